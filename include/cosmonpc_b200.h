/*
 * cosmonpc_b200.h -- C ABI of the B200 mesh-estimator library (libcosmonpc_b200.so).
 *
 * The reference (zhaoruiyang98/CosmoNPC) is pure Python; its mesh path calls
 * pmesh (paint / r2c / c2r), numexpr (Y_lm, Legendre) and numpy (bincount,
 * triple products).  Each entry point below replaces one of those steps and
 * cites the reference lines it stands in for (paths inside the reference
 * project).  Conventions shared by all entry points:
 *
 *  - Every function returns an int status (CNPC_OK = 0) and never throws.
 *  - All pointers named d_* are device pointers owned by the caller; h_*
 *    pointers are host memory read before the function returns.
 *  - Work is enqueued on the given stream; nothing synchronises the host.
 *  - dtype selects the arithmetic: CNPC_F32 (float / float2 fields, FP64
 *    accumulators) or CNPC_F64 (double / double2 fields throughout).
 *  - Real meshes are n*n*n, x slowest, z fastest.  Spectra are the half
 *    spectrum of a real field in cuFFT R2C layout: n*n*(n/2+1) complex,
 *    index (ix, iy, iz), n_x = ix - n*(ix >= n/2) (same for y), n_z = iz.
 *  - A context owns cached cuFFT plans and is not thread-safe; use one
 *    context per host thread.
 */
#ifndef COSMONPC_B200_H
#define COSMONPC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *cnpc_stream_t; /* == cudaStream_t */
typedef struct cnpc_ctx cnpc_ctx;

enum cnpc_status {
    CNPC_OK = 0,
    CNPC_EINVAL = 1,   /* bad argument (maps to ValueError)              */
    CNPC_ENOMEM = 2,   /* device allocation refused (MemoryError)        */
    CNPC_ECUDA = 3,    /* CUDA runtime error                             */
    CNPC_ECUFFT = 4,   /* cuFFT error                                    */
    CNPC_ETIMEOUT = 5  /* a bounded device-side wait gave up             */
};

enum cnpc_dtype { CNPC_F32 = 0, CNPC_F64 = 1 };

/* mass-assignment window order p: NGP 1, CIC 2, TSC 3, PCS 4 */
enum cnpc_window { CNPC_NGP = 1, CNPC_CIC = 2, CNPC_TSC = 3, CNPC_PCS = 4 };

/* k-space window compensation (math_evaluator.py:206-309) */
enum cnpc_comp {
    CNPC_COMP_NONE = 0,
    CNPC_COMP_SINC = 1,      /* v / prod sinc(w/2)^p            me:206-248 */
    CNPC_COMP_SHOTNOISE = 2, /* v / prod sqrt(C_p(sin^2(w/2)))  me:251-275 */
    CNPC_COMP_BKNOISE = 3    /* v * prod C_p / sinc^(2p)        me:278-309 */
};

/* Spherical harmonic descriptor.  Value on a unit vector (x, y, z):
 *   Y = norm * poly(z) * (x + i y)^|m|, conjugated and multiplied by
 *   (-1)^|m| when m < 0; poly has degree l-|m| (coef[0] constant term).
 * origin_re/origin_im: the value used at the k = 0 mode, where the reference
 * evaluates its polynomial at (0, 0, 0) (math_evaluator.py:12-22, :35-131). */
typedef struct cnpc_harmonic {
    int l;
    int m;
    double norm;
    double coef[9];
    double origin_re;
    double origin_im;
} cnpc_harmonic;

/* One real shell field to synthesise (see cnpc_shell_spectra). */
typedef struct cnpc_shell_item {
    int bin;       /* index into the edges: mask = e[bin] <= |k| < e[bin+1]   */
    int harmonic;  /* index into the harmonic table                           */
    int component; /* 0: real part of the complex shell field, 1: imaginary   */
    int source;    /* 0: spectrum A, 1: spectrum B, 2: unit spectrum (=1)     */
    int conj;      /* 1: use conj(Y) instead of Y                             */
} cnpc_shell_item;

#define CNPC_MAX_EDGES 257
#define CNPC_MAX_HARMONICS 16
#define CNPC_MAX_ITEMS 256
#define CNPC_MAX_POLES 8

/* ---------------------------------------------------------------- context */
int cnpc_ctx_create(cnpc_ctx **ctx, int device);
int cnpc_ctx_destroy(cnpc_ctx *ctx);
/* Text of the last error recorded in this context ("" if none). */
const char *cnpc_ctx_last_error(cnpc_ctx *ctx);
const char *cnpc_status_string(int status);
/* Library version as major*10000 + minor*100 + patch. */
int cnpc_version(void);

/* Failure detection of the device-side waits (no counterpart in the
 * reference, which has no device code).  The FP64 contraction kernel
 * (cnpc_contract_gram with CNPC_F64) waits on shared-memory mbarriers for its
 * staged copies; every such wait gives up after `polls` checks (default
 * 4194304, about a second; 0 gives up at the first check, which tests the
 * failure path without hanging anything).  A wait that gives up lets the
 * block drain its own copies, makes that call's outputs NaN and sets the
 * context's status word to CNPC_ETIMEOUT. */
int cnpc_ctx_set_wait_limit(cnpc_ctx *ctx, int64_t polls);
/* Synchronises `stream`, stores the context's status word in *h_status
 * (CNPC_OK, or CNPC_ETIMEOUT when a bounded wait gave up since the previous
 * read) and clears it.  The word is sticky: several calls can be queued
 * before one read. */
int cnpc_ctx_take_status(cnpc_ctx *ctx, cnpc_stream_t stream, int *h_status);

/* ------------------------------------------------------------------ paint
 * Replaces pmesh ParticleMesh.paint as called by pm_painter
 * (src/cosmonpc/mesh_generator.py:172-224, :199, :204-205).
 * h/d_pos: (np, 3) float64 positions; d_weight: np float64 or NULL (weight 1).
 * Zeroes and fills d_mesh (node i at x = i*L/n, window order `window`); when
 * d_mesh_shifted is non-NULL also paints the +1/2-cell interlaced mesh in the
 * same pass (pm.affine.shift(0.5), mesh_generator.py:201-205). */
int cnpc_paint(cnpc_ctx *ctx, int dtype, const double *d_pos, const double *d_weight,
               int64_t np, int n, double boxsize, int window,
               void *d_mesh, void *d_mesh_shifted, cnpc_stream_t stream);

/* cnpc_paint in a shifted frame, with scaled masses, optionally accumulating:
 * grid coordinates (x - h_origin) * n / L (h_origin: 3 host doubles or NULL),
 * masses weight * mass_scale, and the meshes are zeroed first unless
 * `accumulate`.  Replaces pm_painter's Position - boxcenter
 * (mesh_generator.py:182-183) and the x-space scalings of the painted survey
 * fields (mesh_generator.py:449-454, :666-668, :1117-1120), which are linear
 * in the masses. */
int cnpc_paint_ex(cnpc_ctx *ctx, int dtype, const double *d_pos, const double *d_weight,
                  int64_t np, int n, double boxsize, int window, const double *h_origin,
                  double mass_scale, int accumulate, void *d_mesh, void *d_mesh_shifted,
                  cnpc_stream_t stream);

/* --------------------------------------------------------------------- FFT
 * Replace RealField.r2c / ComplexField.c2r of pmesh.  Unnormalised cuFFT
 * transforms of `batch` fields; the 1/n^3 of pmesh's r2c is folded into
 * cnpc_forward_finish.  Spectra of a batch are contiguous; real field b starts
 * at d_real + b * real_dist elements (real_dist 0 means n^3; a padded distance
 * keeps batched fields off power-of-two strides).  c2r may overwrite its input. */
int cnpc_fft_r2c(cnpc_ctx *ctx, int dtype, int n, int batch, const void *d_real,
                 int64_t real_dist, void *d_spec, cnpc_stream_t stream);
int cnpc_fft_c2r(cnpc_ctx *ctx, int dtype, int n, int batch, void *d_spec,
                 void *d_real, int64_t real_dist, cnpc_stream_t stream);

/* Finishes the forward transform in place on d_spec:
 *   c = s1 / n^3                       (d_spec2 == NULL)
 *   c = 0.5 s1/n^3 + 0.5 s2/n^3 e^{i(kx+ky+kz)H/2}  (interlaced combine,
 *                                        mesh_generator.py:211-218)
 *   c *= scale, then the compensation `comp` of window order `window`
 *   (clustering_estimator.py:599-603, :815-816), and the k = 0 mode is set to
 *   k0_value (the reference clears it for pk, ce:634-636, and it equals
 *   (sum w / n^3)/dV - NZ for the bk overdensity, ce:808-816); k0_value NaN
 *   keeps the computed k = 0 mode (survey fields, ce:590-603, ce:1625-1627).
 *   band_kmax > 0 zeroes modes with |k| >= band_kmax. */
int cnpc_forward_finish(cnpc_ctx *ctx, int dtype, int n, double boxsize, void *d_spec,
                        const void *d_spec2, double scale, int comp, int window,
                        double k0_value, double band_kmax, cnpc_stream_t stream);

/* cnpc_forward_finish that also writes the finished spectrum, zeroed at
 * |k| >= band_out_kmax, to d_band_out: the band-limited copy of the
 * overdensity spectrum that the bk_sugi box estimator transforms into G_00
 * (ce:843-851; the triple sums see G_00 only at |k| < 2 k_max).  d_band_out may be d_spec2 (each element is read before it
 * is overwritten); it must not be d_spec. */
int cnpc_forward_finish_band(cnpc_ctx *ctx, int dtype, int n, double boxsize, void *d_spec,
                             const void *d_spec2, double scale, int comp, int window,
                             double k0_value, double band_kmax, void *d_band_out,
                             double band_out_kmax, cnpc_stream_t stream);

/* -------------------------------------------------------- k-bin statistics
 * get_kbin_count (math_evaluator.py:452-481): full-space mode counts and sum
 * of |k| per bin [e_b, e_{b+1}), |k| computed in FP64 as
 * sqrt((kx^2 + ky^2) + kz^2) with k = (2 n) pi / L.  d_counts / d_ksum get
 * nedges-1 doubles each. */
int cnpc_kbin_counts(cnpc_ctx *ctx, int n, double boxsize, const double *h_edges,
                     int nedges, double *d_counts, double *d_ksum, cnpc_stream_t stream);

/* Power-spectrum shell sums for calculate_power_spectrum_box
 * (clustering_estimator.py:638-693): for each pole l in h_poles,
 *   sum_{k in bin} (Re a Re b + Im a Im b) * P_l(khat . los)
 * over full k-space (half spectrum times multiplicity), FP64 accumulators.
 * d_spec_b may equal d_spec_a.  d_sums: npoles * (nedges-1) doubles. */
int cnpc_pk_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                 const void *d_spec_b, const double *h_edges, int nedges,
                 const int *h_poles, int npoles, const double *h_los, double *d_sums,
                 cnpc_stream_t stream);

/* Shot-noise shell sums for calculate_bk_sugi_box (ce:1405-1434) and the
 * S3-FFT source spectrum (ce:1187-1210):
 *   P(k) = V^2 a(k) conj(b(k)) - sn0 * W_bknoise(k)
 *   d_sums[2*bin] = sum_{bin} Re P(k) * Y_L0(khat)   (FP64; d_sums[2*bin+1] = 0)
 * with harmonic h_yl0 (NULL: 1): half-spectrum modes carry their full-space
 * multiplicity, so the real part is the full-space sum for even L.  If d_source is non-NULL, P(k) (without Y)
 * is also written there, zeroed at |k| >= band_kmax when band_kmax > 0, and
 * d_sums[2*(nedges-1)] receives the full-space sum of that source (its value
 * at x = 0 after the c2r), so d_sums then holds nedges pairs. */
int cnpc_sn_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                 const void *d_spec_b, double volume_sq, double sn0, int window,
                 const cnpc_harmonic *h_yl0, const double *h_edges, int nedges,
                 double *d_sums, void *d_source, double band_kmax, cnpc_stream_t stream);

/* cnpc_sn_bins for ncfg = 1 or 2 configurations of the bk_sugi box loop over
 * angular configurations (ce:1187-1210, :1405-1434) in one pass over the
 * modes: configuration c has its own sn0 h_sn0[c], harmonic h_yl0[c] (NULL:
 * 1), d_sums[c] and d_source[c] (NULL: no source), each with the layout and
 * meaning of cnpc_sn_bins; the spectra, volume_sq, window, edges and
 * band_kmax are shared. */
int cnpc_sn_bins_multi(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                       const void *d_spec_b, double volume_sq, int window, int ncfg,
                       const double *h_sn0, const cnpc_harmonic *const *h_yl0,
                       const double *h_edges, int nedges, double *const *d_sums,
                       void *const *d_source, double band_kmax, cnpc_stream_t stream);

/* Shell spectra: replaces (ylm_weighted_cfield * mask_i) before .c2r() in
 * clustering_estimator.py:898-969, :1012-1050, :1215-1219.  For each item j,
 * writes half spectrum j of d_out (n*n*(n/2+1) complex each):
 *   src(k) * mask_bin(|k|) * phi(k)
 * where the complex shell field F = c2r(src * Y * mask) is split into real
 * fields Re F = c2r(src * phi_re), Im F = c2r(src * phi_im) with
 *   even l: phi_re = Re Y,   phi_im = Im Y
 *   odd l:  phi_re = i Im Y, phi_im = -i Re Y
 * (valid because src is Hermitian on |k| < k_Nyquist). */
int cnpc_shell_spectra(cnpc_ctx *ctx, int dtype, int n, double boxsize,
                       const void *d_spec_a, const void *d_spec_b,
                       const double *h_edges, int nedges,
                       const cnpc_harmonic *h_harmonics, int nharmonics,
                       const cnpc_shell_item *h_items, int nitems, void *d_out,
                       cnpc_stream_t stream);

/* ------------------------------------------------------------ survey path
 * Survey catalogs arrive as the raw big-endian rows of a FITS binary table
 * (catalog_processor.py:128-183 reads them with fitsio); one call decodes the
 * columns the reference uses on the device. */
enum cnpc_coltype {
    CNPC_CT_ABSENT = 0, CNPC_CT_F64 = 1, CNPC_CT_F32 = 2, CNPC_CT_I16 = 3,
    CNPC_CT_I32 = 4, CNPC_CT_I64 = 5, CNPC_CT_U8 = 6, CNPC_CT_BOOL = 7
};
/* one scalar FITS column: value = zero + scale * raw (TZEROn / TSCALn) */
typedef struct cnpc_column {
    int type;    /* cnpc_coltype                     */
    int offset;  /* byte offset of the column in a row */
    double scale;
    double zero;
} cnpc_column;
enum cnpc_colid {
    CNPC_COL_RA = 0, CNPC_COL_DEC, CNPC_COL_Z, CNPC_COL_WEIGHT, CNPC_COL_SYSTOT,
    CNPC_COL_NOZ, CNPC_COL_CP, CNPC_COL_FKP, CNPC_COL_NZ, CNPC_NCOLS
};
/* completeness weight (add_completeness_weight, catalog_processor.py:186-290):
 * COLUMN: the WEIGHT slot (an existing WEIGHT column or the alias column);
 * ONE: 1; BOSS: SYSTOT (NOZ + CP - 1); EBOSS: SYSTOT NOZ CP */
enum cnpc_weight_rule { CNPC_W_COLUMN = 0, CNPC_W_ONE = 1, CNPC_W_BOSS = 2, CNPC_W_EBOSS = 3 };
typedef struct cnpc_catalog_spec {
    int64_t row_bytes;
    cnpc_column col[CNPC_NCOLS]; /* NZ slot: the NZ or NX column, or absent (NZ = 1) */
    int weight_rule;
    int has_zrange;              /* keep rows with z_min < Z < z_max (cp:506-508) */
    double z_min, z_max;
    double h, omega_m;           /* flat LCDM, no radiation (cp:617-632)          */
    int cosmology;               /* CNPC_COSMO_FLAT_LCDM: (h, omega_m);
                                    CNPC_COSMO_PLANCK18: the fallback of cp:610-625
                                    when the config gives h but no Omega0:
                                    astropy's Planck18 (H0 67.66, Om0 0.30966,
                                    Tcmb0 2.7255 K, Neff 3.046, one 0.06 eV
                                    neutrino), distances times the config's h;
                                    omega_m is ignored */
} cnpc_catalog_spec;
enum cnpc_cosmology { CNPC_COSMO_FLAT_LCDM = 0, CNPC_COSMO_PLANCK18 = 1 };

/* ------------------------------------------------------------ box catalogs
 * Box catalogs in FITS or HDF5 files (catalog_processor.py:388-445).  A
 * column is a strided run of scalars in device memory: the raw rows of a FITS
 * binary table (big_endian = 1, stride = the row size, d_base = rows + column
 * offset) or one contiguous HDF5 dataset (stride = the element size). */
typedef struct cnpc_colref {
    const void *d_base; /* value of row 0; unused when type is CNPC_CT_ABSENT */
    int64_t stride;     /* bytes between consecutive rows                      */
    int type;           /* cnpc_coltype                                        */
    int big_endian;
    double scale;       /* value = zero + scale * raw                          */
    double zero;
} cnpc_colref;
enum cnpc_box_colid {
    CNPC_BOX_X = 0, CNPC_BOX_Y, CNPC_BOX_Z, CNPC_BOX_VX, CNPC_BOX_VY, CNPC_BOX_VZ, CNPC_BOX_W, CNPC_BOX_NCOLS
};

/* Decode a box catalog: d_pos (nrows, 3) from the X/Y/Z columns (absent:
 * 0, as the reference leaves Position zero when no position columns match),
 * d_weight from the W column (absent: 1).  With apply_rsd, the shift of
 * add_rsd (catalog_processor.py:648-693, box branch) is applied on the device:
 * x_d = (x_d + h_shift[d] * v_d) mod box_length with h_shift[d] =
 * rsd_factor * los_d (the reference multiplies los and the velocity
 * elementwise) and numpy's float remainder; the velocity columns must exist. */
int cnpc_box_catalog(cnpc_ctx *ctx, int64_t nrows, const cnpc_colref *h_cols, int apply_rsd,
                     const double *h_shift, double box_length, double *d_pos, double *d_weight,
                     cnpc_stream_t stream);

/* Decode, z-cut and convert a survey catalog: catalog_reader's survey branch
 * (catalog_processor.py:493-586) with ra_dec_z_to_xyz (cp:589-645).
 * Kept rows are written in file order to d_pos (n, 3), d_weight, d_wfkp, d_nz;
 * the buffers must hold nrows entries.  Positions are D_C(z) h (cos d cos a,
 * cos d sin a, sin d) in Mpc/h with D_C from 16-point Gauss-Legendre panels.
 * The call waits for the stream to return the kept count in *h_kept. */
int cnpc_catalog_decode(cnpc_ctx *ctx, const void *d_rows, int64_t nrows,
                        const cnpc_catalog_spec *h_spec, double *d_pos, double *d_weight,
                        double *d_wfkp, double *d_nz, int64_t *h_kept, cnpc_stream_t stream);

/* Per-particle sums of compute_particle_sums_pk / _bk (mesh_generator.py:1131-1268)
 * and the position range of catalog_reader's boxcenter (cp:564-574).  d_out:
 *   [0] sum w wfkp   [1] sum w   [2] sum w nz wfkp^2   [3] sum (w wfkp)^2
 *   [4] sum nz^2 w^2 wfkp^3,
 *   [5 + 2q], [6 + 2q]: re, im of sum (w wfkp)^3 conj(Y_q(x/|x|)) for the
 *   nharm harmonics h_ylm (S_LM), then min x, y, z and max x, y, z. */
#define CNPC_PSUM_COUNT 5
int cnpc_particle_sums(cnpc_ctx *ctx, int64_t np, const double *d_pos, const double *d_weight,
                       const double *d_wfkp, const double *d_nz, const cnpc_harmonic *h_ylm,
                       int nharm, double *d_out, cnpc_stream_t stream);

/* d_out[i] = (w[i] wfkp[i])^power, power 1 (paint weights, mg:422-445) or 2
 * (the N-field weights of get_N_field, mg:1082-1083). */
int cnpc_catalog_weights(cnpc_ctx *ctx, int64_t np, const double *d_weight, const double *d_wfkp,
                         int power, double *d_out, cnpc_stream_t stream);

/* The reference holds an interlaced painted field as the complex-to-complex
 * c2r of c = s1/2 + s2/2 e^{i k.H/2} (mesh_generator.py:207-219); on the
 * Nyquist planes c is not Hermitian, so the field has an imaginary part.
 * This writes, from the raw R2C spectra s1, s2 (s1 / n^3 is pmesh's r2c),
 *   d_herm = scale * (c(k) + conj c(-k)) / 2        (c2r -> Re field)
 *   d_anti = scale * (-i) (c(k) - conj c(-k)) / 2   (c2r -> Im field)
 * with the reference's index convention (index i >= n/2 is k = (i - n) 2pi/L
 * on every axis).  d_spec2 NULL: d_herm = scale * s1 / n^3, d_anti unused.
 * accumulate adds to d_herm / d_anti; in place (d_herm == d_spec,
 * d_anti == d_spec2) is allowed without accumulate. */
int cnpc_interlace_split(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec,
                         const void *d_spec2, double scale, int accumulate, void *d_herm,
                         void *d_anti, cnpc_stream_t stream);

/* x-space harmonic weighting of a complex field F = re + i im (im may be NULL):
 *   out_re + i out_im = scale * F(x) * Y(xhat)   (conj: conj(Y))
 * at the cell positions of get_xgrid (math_evaluator.py:25-32): the node
 * coordinate i L / n wrapped into [-L/2, L/2), plus L / (2 n) + boxcenter.
 * Replaces rfield * Y_lm(xgrid) in ce:3118-3124, ce:1700-1703, ce:2262, ce:2346,
 * ce:2496.  d_out_im may be NULL when the product is known to be real. */
int cnpc_xspace_harmonic(cnpc_ctx *ctx, int dtype, int n, double boxsize, const double *h_boxcenter,
                         const void *d_re, const void *d_im, const cnpc_harmonic *h_y, int conj,
                         double scale, void *d_out_re, void *d_out_im, cnpc_stream_t stream);

/* A spectral operand of the survey sums: Hermitian half spectrum p (q NULL),
 * or X = P + i Q for the non-Hermitian FFT of a complex field whose real and
 * imaginary parts have half spectra P and Q (X(-k) = conj P + i conj Q).
 * p NULL (and q NULL) is the unit spectrum.  The operand's value is
 * scale * comp(k) * (p, X or 1). */
typedef struct cnpc_operand {
    const void *p;
    const void *q;
    double scale;
    int comp;
} cnpc_operand;

/* Complex shell sums over full k-space, d_sums[2 b + {0, 1}]:
 *   sum_{k in bin b} weight * (U(k) conj V(k) - sbar W_bknoise(k)) * Z(khat)
 * Z = Y of h_z (conj_z: conj Y; NULL: 1; Y(-khat) = (-1)^l Y(khat)).
 * Replaces radial_binning of the survey terms: a conj G_l (ce:456-468 with
 * get_G_ell ce:3104-3134), the S1 field (ce:2254-2296) and Q_L (ce:2338-2385). */
int cnpc_survey_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, int window,
                     const cnpc_operand *u, const cnpc_operand *v, double sbar_re, double sbar_im,
                     const cnpc_harmonic *h_z, int conj_z, double weight, const double *h_edges,
                     int nedges, double *d_sums, cnpc_stream_t stream);

/* The S3-FFT source spectrum src = U conj V - sbar W_bknoise (ce:2484-2511)
 * split like cnpc_interlace_split into its Hermitian part (d_herm, c2r ->
 * Re src) and -i times its anti-Hermitian part (d_anti, c2r -> Im src),
 * zero at |k| >= band_kmax when band_kmax > 0. */
int cnpc_survey_source(cnpc_ctx *ctx, int dtype, int n, double boxsize, int window,
                       const cnpc_operand *u, const cnpc_operand *v, double sbar_re, double sbar_im,
                       double band_kmax, void *d_herm, void *d_anti, cnpc_stream_t stream);

/* d_out(k) += weight * (Y(khat) X(k) + conj(Y(-khat) X(-k))) / 2: the
 * Hermitian part of Y X for the operand x (a half spectrum, accumulated).
 * Summed over m with the weights of get_G_ell it gives the fast-mode fields
 * F_l = (G_l + conj G_l(-k)) / 2 of ce:402-417 without the space-inversion
 * exchange of math_evaluator.py:806-977. */
int cnpc_survey_hermitian_accumulate(cnpc_ctx *ctx, int dtype, int n, double boxsize, int window,
                                     const cnpc_operand *x, const cnpc_harmonic *h_y, double weight,
                                     void *d_out, cnpc_stream_t stream);

/* d_out[0] + i d_out[1] = sum_x prod_{j < nf} (re_j(x) + i im_j(x)), nf 1..3,
 * h_re / h_im: host arrays of nf device pointers (h_im or its entries may be
 * NULL).  Replaces the normalisation sums np.sum(D * R) and friends
 * (mesh_generator.py:503-519, :829-830, :903-905, :961-990). */
int cnpc_field_product_sum(cnpc_ctx *ctx, int dtype, int64_t ncell, int nf, const void *const *h_re,
                           const void *const *h_im, double *d_out, cnpc_stream_t stream);

/* d_out = a x + b y over ncell real cells (d_y may be NULL); the x-space
 * combinations rfield_data - alpha rfield_randoms (mg:449-454, :666-668). */
int cnpc_field_axpby(cnpc_ctx *ctx, int dtype, int64_t ncell, double a, const void *d_x, double b,
                     const void *d_y, void *d_out, cnpc_stream_t stream);

/* Parity fold of a weight field for sums over fields of definite parity.
 * When F_a(-x) F_b(-x) = sign F_a(x) F_b(x) on the grid (shell fields of the
 * unit spectrum, conj(Y_lm) times a shell mask, have the parity (-1)^l, so a
 * product of two has sign (-1)^(l_a + l_b)),
 *   sum_x G F_a F_b = sum over the planes x = 0 .. n/2 of G' F_a F_b,
 * G'[x][y][z] = G[x][y][z] on the planes 0 and n/2 and
 * G[x][y][z] + sign G[n - x][-y][-z] (indices mod n) on the others.
 * d_out holds (n/2 + 1) n^2 cells: the contraction then runs over
 * ncell = (n/2 + 1) n^2 with the fields' first planes (x is the slowest
 * index).  The FFT S3 sums np.sum(S3_field * F1 * F2)
 * (clustering_estimator.py:1257, :1341) thus read half of every field. */
int cnpc_field_parity_fold(cnpc_ctx *ctx, int dtype, int n, const void *d_in, int sign, void *d_out,
                           cnpc_stream_t stream);

/* Shell fields in one call, FP32: the real fields
 *   h_out_fields[j] = c2r(src * Y * mask_bin * phi)   (item j, as in
 * cnpc_shell_spectra followed by cnpc_fft_c2r) for n = 64, 128, 192 or 256, when
 * every item's bin lies below k = (n/4) 2 pi / L -- always the case for the
 * bispectrum shells, whose top edge k_max is below k_Nyquist / 2 by the
 * reference's own check (task_executor.py:192-196).  The inverse FFT runs on
 * the band only (x pass on the in-band columns, then y and z per x-slab in
 * shared memory) and each field is written once.  Output fields are n^3
 * floats, 16-byte aligned; h_out_fields is a host array of nitems device
 * pointers. */
int cnpc_shell_fields(cnpc_ctx *ctx, int n, double boxsize, const void *d_spec_a,
                      const void *d_spec_b, const double *h_edges, int nedges,
                      const cnpc_harmonic *h_harmonics, int nharmonics,
                      const cnpc_shell_item *h_items, int nitems, void *const *h_out_fields,
                      cnpc_stream_t stream);

/* ------------------------------------------------------ x-space reductions
 * Replaces np.sum(G * F1 * F2) of clustering_estimator.py:972, :1051, :1257,
 * :1341 for real component fields.
 * Gram form: d_out[i*nb + j] = sum_x G(x) F_{a_i}(x) F_{b_j}(x), FP64 result,
 * where field f starts at d_fields + f * field_stride (elements).
 * Per-block partials live in the context's scratch buffer, so calls on one
 * context must not overlap on different streams. */
int cnpc_contract_gram(cnpc_ctx *ctx, int dtype, int64_t ncell, const void *d_g,
                       const void *d_fields, int64_t field_stride,
                       const int *h_a, int na, const int *h_b, int nb, double *d_out,
                       cnpc_stream_t stream);

/* FP32 Gram with several weight fields in one launch: d_out[i*nb + j] =
 * sum_x G_{h_ag[i]}(x) F_{h_a[i]}(x) F_{h_b[j]}(x), where h_gs[0..ngs) (ngs <= 4) are
 * device pointers to the weight fields and h_ag gives each row's weight; na <= 48,
 * nb <= 24, and ngs + na (padded to 8) + nb (padded to 4, omitted when the columns
 * are a run of the rows) <= 48 staged rows.  The FFT S3 sums of several angular configurations share their unit
 * shell fields (clustering_estimator.py:1257, :1341) and are contracted together. */
int cnpc_contract_gram_multi_g(cnpc_ctx *ctx, int64_t ncell, const float *const *h_gs, int ngs,
                               const float *d_fields, int64_t field_stride, const int *h_a,
                               const int *h_ag, int na, const int *h_b, int nb, double *d_out,
                               cnpc_stream_t stream);

/* Pair-list form: d_out[p] = sum_x G(x) F_{h_a[p]}(x) F_{h_b[p]}(x), p < npairs
 * (<= 256), FP64 result; the diagonal data vector's same-bin pairs
 * (clustering_estimator.py:998-1061, :1983-2035) without the whole Gram block.
 * ncell and field_stride multiples of 4; G and fields aligned to 4 elements. */
int cnpc_contract_pairs(cnpc_ctx *ctx, int dtype, int64_t ncell, const void *d_g,
                        const void *d_fields, int64_t field_stride, const int *h_a,
                        const int *h_b, int npairs, double *d_out, cnpc_stream_t stream);

/* FP32 Gram contraction on the tensor cores: d_out[i*nb + j] =
 * sum_x G F_{h_a[i]} F_{h_b[j]} for na <= 40 rows and nb <= 24 columns, the
 * same sums as cnpc_contract_gram (clustering_estimator.py:911-981,
 * :1983-2035).  tcgen05.mma kind::tf32 with each FP32 operand split into a
 * TF32 hi/lo pair (all four products in one M = 128, N = 48 MMA per 8 cells;
 * the A operand G F_a in tensor memory, written from registers, the B
 * operand F_b in 128-byte-swizzled shared memory), FP32 accumulators folded
 * into FP64 every 512 cells; product error ~2^-22 relative.  ncell and
 * field_stride are multiples of 4; G and fields 16-byte aligned.  Its
 * bounded waits report through the context's status word
 * (cnpc_ctx_take_status). */
int cnpc_contract_gram_tc(cnpc_ctx *ctx, int64_t ncell, const float *d_g, const float *d_fields,
                          int64_t field_stride, const int *h_a, int na, const int *h_b, int nb,
                          double *d_out, cnpc_stream_t stream);

/* cnpc_contract_gram_tc with a weight field per row, in one launch:
 * d_out[i*nb + j] = sum_x G_{h_ag[i]} F_{h_a[i]} F_{h_b[j]}, ngs <= 4 weight
 * fields h_gs[0..ngs-1] (device pointers, 16-byte aligned).  The FFT S3 sums
 * of several angular configurations contract their own source fields with
 * the same unit-spectrum shells (clustering_estimator.py:1182-1384). */
int cnpc_contract_gram_tc_multi_g(cnpc_ctx *ctx, int64_t ncell, const float *const *h_gs, int ngs,
                                  const float *d_fields, int64_t field_stride, const int *h_a,
                                  const int *h_ag, int na, const int *h_b, int nb, double *d_out,
                                  cnpc_stream_t stream);

/* Allocation-free form of cnpc_contract_gram.  It has no counterpart in the
 * reference; it exists for callers that must not have a library allocate
 * device memory, such as an application whose own pool owns the whole device,
 * or one that cannot afford the device-wide synchronisation cudaFree may
 * cause.  It takes no context and calls no cudaMalloc, cudaFree or allocating
 * library routine: the per-block partial sums live in one fixed 8 MiB array in
 * the library's device memory, which every GPU that loads the library holds
 * until the process exits.  The caller still owns G, the fields and d_out.
 *  - Limits per call: CNPC_F32 at most 48 rows x 24 columns with
 *    1 + pad8(na) [+ pad4(nb) when b is not a contiguous run of a whose
 *    padded window stays inside a's] <= 48 staged rows (so 40 x 24 with b
 *    inside a, or 24 x 20 with b separate); CNPC_F64 at most 128 x 128 with
 *    1 + pad8(na) [+ pad4(nb) likewise] <= 110 staged rows.  Larger calls, or
 *    misaligned fields (16-byte base, field_stride and ncell), return
 *    CNPC_EINVAL.
 *  - The array bounds the grid: FP32 windows above about 24 x 12 outputs run
 *    fewer blocks than cnpc_contract_gram (e.g. 163 instead of 2 per SM at
 *    40 x 20), so they take longer than the regular call.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) and caches it; make that first call before any
 *    stream capture.  The cached address belongs to the device's primary
 *    context: after cudaDeviceReset (or any teardown of that context) it is
 *    stale, so do not call this entry point again in that process.
 *  - A bounded device wait of the FP64 kernel that gives up (see
 *    cnpc_ctx_set_wait_limit; here the default limit) is reported only
 *    through NaN in d_out, since there is no context to hold a status word.
 *  - All calls share the array, so calls whose work overlaps on the GPU (on
 *    different streams, or from different threads) race and corrupt each
 *    other's partial sums: serialise them. */
int cnpc_contract_gram_noalloc(int dtype, int64_t ncell, const void *d_g, const void *d_fields,
                               int64_t field_stride, const int *h_a, int na, const int *h_b, int nb,
                               double *d_out, cnpc_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* COSMONPC_B200_H */
