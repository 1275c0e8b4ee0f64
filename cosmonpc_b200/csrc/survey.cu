// Survey-geometry stages: FITS rows decoded on the device (z cut, completeness
// weight, RA/DEC/Z -> comoving Cartesian), per-particle sums, the complex
// "real" fields of an interlaced paint split into real and imaginary parts,
// x-space spherical-harmonic weighting, and the shell sums / source spectra of
// the survey estimators.
#include <cmath>
#include <cstring>
#include <vector>

#include "bins.cuh"

namespace cnpc {

// ----------------------------------------------------------------- catalogs
struct Gauss16 {
    double x[16];
    double w[16];
};

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_16).
static Gauss16 gauss_legendre16() {
    Gauss16 g;
    const int n = 16;
    for (int i = 0; i < n; ++i) {
        double x = std::cos(kPi * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (x * p1 - p0) / (x * x - 1.0);
            const double dx = p1 / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        g.x[i] = x;
        g.w[i] = 2.0 / ((1.0 - x * x) * dp * dp);
    }
    return g;
}

struct CatalogParams {
    int64_t row_bytes;
    cnpc_column col[CNPC_NCOLS];
    int weight_rule;
    int has_zrange;
    double z_min, z_max;
    double omega_m;
    double h;
    double hubble_distance;  // c / H0 in Mpc
    int planck18;            // E(z) with photons and a massive neutrino (Planck18Radiation)
    double ogamma0, ode0, nu_prefac, nu_y, nu_massless;
    Gauss16 gl;
};

// astropy's Planck18 realisation (H0 = 67.66 km/s/Mpc, Om0 = 0.30966,
// Tcmb0 = 2.7255 K, Neff = 3.046, m_nu = (0, 0, 0.06) eV, flat), restated
// from astropy's published FLRW formulas with CODATA 2018 constants:
//   Ogamma0 = (4 sigma_SB / c^3) Tcmb0^4 / rho_crit0, rho_crit0 = 3 H0^2 / (8 pi G);
//   the neutrino density relative to photons, for neutrinos of y = m c^2 / (k_B T_nu0)
//   with T_nu0 = (4/11)^(1/3) Tcmb0 (Komatsu et al. 2011, eq. 26 fit),
//   n(z) = (7/8)(4/11)^(4/3) (Neff / 3) [sum (1 + (0.3173 y / (1+z))^1.83)^(1/1.83) + N_massless];
//   E(z)^2 = (1+z)^2 ((Or (1+z) + Om0) (1+z)) + Ode0, Or = Ogamma0 (1 + n(z)),
//   Ode0 = 1 - Om0 - Ogamma0 - Ogamma0 n(0).
struct Planck18Radiation {
    double ogamma0, ode0, nu_prefac, nu_y, nu_massless, hubble_distance;
};
static Planck18Radiation planck18_radiation() {
    const double pi = 3.14159265358979323846;
    const double sigma_sb = 5.670374419e-8, c = 299792458.0, G = 6.67430e-11;
    const double kB_eV = 1.380649e-23 / 1.602176634e-19;
    const double mpc = 3.0856775814913673e22;
    const double H0 = 67.66, Tcmb0 = 2.7255, Neff = 3.046, m_nu = 0.06;
    const double h0_si = H0 * 1000.0 / mpc;
    const double rho_crit = 3.0 * h0_si * h0_si / (8.0 * pi * G);
    Planck18Radiation r;
    r.ogamma0 = (4.0 * sigma_sb / (c * c * c)) * Tcmb0 * Tcmb0 * Tcmb0 * Tcmb0 / rho_crit;
    const double tnu0 = 0.7137658555036082 * Tcmb0;
    r.nu_y = m_nu / (kB_eV * tnu0);
    r.nu_prefac = 0.22710731766 * (Neff / 3.0);
    r.nu_massless = 2.0;
    const double n0 = r.nu_prefac * (std::pow(1.0 + std::pow(0.3173 * r.nu_y, 1.83), 0.54644808743) + r.nu_massless);
    r.ode0 = 1.0 - 0.30966 - r.ogamma0 - r.ogamma0 * n0;
    r.hubble_distance = c / 1000.0 / H0;
    return r;
}

__device__ inline double read_column(const uint8_t *row, const cnpc_column &c) {
    const uint8_t *p = row + c.offset;
    int nb = 8;
    switch (c.type) {
        case CNPC_CT_F32: case CNPC_CT_I32: nb = 4; break;
        case CNPC_CT_I16: nb = 2; break;
        case CNPC_CT_U8: case CNPC_CT_BOOL: nb = 1; break;
        default: nb = 8;
    }
    uint64_t u = 0;
    for (int i = 0; i < nb; ++i) u = (u << 8) | (uint64_t)p[i];
    double v;
    switch (c.type) {
        case CNPC_CT_F64: v = __longlong_as_double((long long)u); break;
        case CNPC_CT_F32: v = (double)__int_as_float((int)(uint32_t)u); break;
        case CNPC_CT_I16: v = (double)(int16_t)(uint16_t)u; break;
        case CNPC_CT_I32: v = (double)(int32_t)(uint32_t)u; break;
        case CNPC_CT_I64: v = (double)(long long)u; break;
        case CNPC_CT_U8: v = (double)u; break;
        case CNPC_CT_BOOL: v = (u == (uint64_t)'T') ? 1.0 : 0.0; break;
        default: v = 0.0;
    }
    if (c.scale != 1.0 || c.zero != 0.0) v = c.zero + c.scale * v;
    return v;
}

__device__ inline bool row_kept(const uint8_t *row, const CatalogParams &p) {
    if (!p.has_zrange) return true;
    const double z = read_column(row, p.col[CNPC_COL_Z]);
    return z > p.z_min && z < p.z_max;
}

// int_0^z dz' / sqrt(Om (1+z')^3 + 1 - Om): 16-point Gauss-Legendre on panels
// of width <= 0.25 (the integrand is analytic well beyond each panel, so the
// rule is exact to rounding).
__device__ inline double los_integral(double z, const CatalogParams &p) {
    const int panels = max(1, (int)ceil(fabs(z) / 0.25));
    const double hw = 0.5 * z / panels;
    const double ol = 1.0 - p.omega_m;
    double sum = 0.0;
    for (int k = 0; k < panels; ++k) {
        const double mid = (2 * k + 1) * hw;
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const double a = 1.0 + (mid + hw * p.gl.x[j]);
            double e2;
            if (p.planck18) {
                const double nrel = p.nu_prefac * (pow(1.0 + pow(0.3173 * p.nu_y / a, 1.83), 0.54644808743) +
                                                   p.nu_massless);
                const double o_r = p.ogamma0 * (1.0 + nrel);
                e2 = a * a * ((o_r * a + p.omega_m) * a) + p.ode0;
            } else {
                e2 = p.omega_m * (a * a * a) + ol;
            }
            s += p.gl.w[j] / sqrt(e2);
        }
        sum += s * hw;
    }
    return sum;
}

constexpr int kRowsPerBlock = 4096;

__global__ void catalog_count_kernel(const uint8_t *rows, int64_t nrows, CatalogParams p, int *counts) {
    const int64_t r0 = (int64_t)blockIdx.x * kRowsPerBlock;
    const int64_t r1 = min(nrows, r0 + kRowsPerBlock);
    int c = 0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) c += row_kept(rows + r * p.row_bytes, p) ? 1 : 0;
    for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += ws[i];
        counts[blockIdx.x] = t;
    }
}

// exclusive scan of counts[0..nb) into offsets[0..nb] (one block)
__global__ void block_scan_kernel(const int *counts, int nb, long long *offsets) {
    __shared__ long long part[1024];
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(nb, b + per);
    long long s = 0;
    for (int i = b; i < e; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long run = 0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            const long long v = part[i];
            part[i] = run;
            run += v;
        }
        offsets[nb] = run;
    }
    __syncthreads();
    long long run = part[threadIdx.x];
    for (int i = b; i < e; ++i) {
        offsets[i] = run;
        run += counts[i];
    }
}

__global__ void catalog_decode_kernel(const uint8_t *rows, int64_t nrows, CatalogParams p,
                                      const long long *offsets, double *pos, double *w, double *wfkp,
                                      double *nz) {
    constexpr double kDeg = kPi / 180.0;
    __shared__ int wc[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int64_t r0 = (int64_t)blockIdx.x * kRowsPerBlock;
    const int64_t r1 = min(nrows, r0 + kRowsPerBlock);
    long long base = offsets[blockIdx.x];
    for (int64_t rb = r0; rb < r1; rb += blockDim.x) {
        const int64_t r = rb + threadIdx.x;
        const uint8_t *row = rows + r * p.row_bytes;
        const bool keep = r < r1 && row_kept(row, p);
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wc[warp] = __popc(bal);
        __syncthreads();
        long long off = base;
        int total = 0;
        for (int i = 0; i < nwarps; ++i) {
            if (i < warp) off += wc[i];
            total += wc[i];
        }
        off += __popc(bal & ((1u << lane) - 1u));
        if (keep) {
            const double ra = __dmul_rn(read_column(row, p.col[CNPC_COL_RA]), kDeg);
            const double dec = __dmul_rn(read_column(row, p.col[CNPC_COL_DEC]), kDeg);
            const double z = read_column(row, p.col[CNPC_COL_Z]);
            const double d = __dmul_rn(__dmul_rn(los_integral(z, p), p.hubble_distance), p.h);
            const double dc = __dmul_rn(d, cos(dec));
            pos[3 * off + 0] = __dmul_rn(dc, cos(ra));
            pos[3 * off + 1] = __dmul_rn(dc, sin(ra));
            pos[3 * off + 2] = __dmul_rn(d, sin(dec));
            double wt = 1.0;
            if (p.weight_rule == CNPC_W_COLUMN) {
                wt = read_column(row, p.col[CNPC_COL_WEIGHT]);
            } else if (p.weight_rule == CNPC_W_BOSS) {
                const double sys = read_column(row, p.col[CNPC_COL_SYSTOT]);
                const double noz = read_column(row, p.col[CNPC_COL_NOZ]);
                const double cp = read_column(row, p.col[CNPC_COL_CP]);
                wt = __dmul_rn(sys, __dsub_rn(__dadd_rn(noz, cp), 1.0));
            } else if (p.weight_rule == CNPC_W_EBOSS) {
                const double sys = read_column(row, p.col[CNPC_COL_SYSTOT]);
                const double noz = read_column(row, p.col[CNPC_COL_NOZ]);
                const double cp = read_column(row, p.col[CNPC_COL_CP]);
                wt = __dmul_rn(__dmul_rn(sys, noz), cp);
            }
            w[off] = wt;
            wfkp[off] = read_column(row, p.col[CNPC_COL_FKP]);
            nz[off] = p.col[CNPC_COL_NZ].type == CNPC_CT_ABSENT ? 1.0 : read_column(row, p.col[CNPC_COL_NZ]);
        }
        base += total;
        __syncthreads();
    }
}

// ------------------------------------------------------------ particle sums
constexpr int kPsumBlocks = 592;
constexpr int kPsumThreads = 256;

struct YlmSet {
    int n;
    cnpc_harmonic h[CNPC_MAX_HARMONICS];
};

// block partials: [CNPC_PSUM_COUNT + 2 * nharm] sums, then 3 minima, 3 maxima
__global__ void particle_sums_kernel(int64_t np, const double *pos, const double *w, const double *wfkp,
                                     const double *nz, YlmSet ylm, double *partial) {
    const int nsum = CNPC_PSUM_COUNT + 2 * ylm.n;
    __shared__ cnpc_harmonic s_h[CNPC_MAX_HARMONICS];  // read at run-time indices
    for (int q = threadIdx.x; q < ylm.n; q += blockDim.x) s_h[q] = ylm.h[q];
    __syncthreads();
    double acc[CNPC_PSUM_COUNT + 2 * CNPC_MAX_HARMONICS];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < nsum; ++i) acc[i] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        const double wi = w[i], fi = wfkp[i], ni = nz[i];
        const double wf = wi * fi;
        acc[0] += wf;
        acc[1] += wi;
        acc[2] += ((wi * ni) * fi) * fi;
        acc[3] += wf * wf;
        acc[4] += ((ni * ni) * (wi * wi)) * (fi * fi * fi);
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        lo[0] = fmin(lo[0], x), lo[1] = fmin(lo[1], y), lo[2] = fmin(lo[2], z);
        hi[0] = fmax(hi[0], x), hi[1] = fmax(hi[1], y), hi[2] = fmax(hi[2], z);
        if (ylm.n) {
            const double r = sqrt(__dadd_rn(__dadd_rn(x * x, y * y), z * z));
            const double xh = x / r, yh = y / r, zh = z / r;
            const double w3 = wf * wf * wf;
            for (int q = 0; q < ylm.n; ++q) {
                const double2 yv = harmonic_eval<double>(s_h[q], xh, yh, zh, false);
                acc[CNPC_PSUM_COUNT + 2 * q] += w3 * yv.x;
                acc[CNPC_PSUM_COUNT + 2 * q + 1] -= w3 * yv.y;  // conj(Y)
            }
        }
    }
    __shared__ double red[kPsumThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < nsum + 6; ++q) {
        double v = q < nsum ? acc[q] : (q < nsum + 3 ? lo[q - nsum] : hi[q - nsum - 3]);
        for (int o = 16; o >= 1; o >>= 1) {
            const double u = __shfl_xor_sync(0xffffffffu, v, o);
            v = q < nsum ? v + u : (q < nsum + 3 ? fmin(v, u) : fmax(v, u));
        }
        if (lane == 0) red[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = red[0];
            for (int i = 1; i < (int)(blockDim.x >> 5); ++i)
                t = q < nsum ? t + red[i] : (q < nsum + 3 ? fmin(t, red[i]) : fmax(t, red[i]));
            partial[(int64_t)q * gridDim.x + blockIdx.x] = t;
        }
        __syncthreads();
    }
}

// reduce the partials of each quantity in a fixed order (one warp per quantity)
__global__ void partials_reduce_kernel(const double *partial, int nblocks, int nsum, int nminmax, double *out) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nsum + nminmax) return;
    const bool is_min = q >= nsum && q < nsum + nminmax / 2;
    const bool is_max = q >= nsum + nminmax / 2;
    double v = is_min ? INFINITY : (is_max ? -INFINITY : 0.0);
    for (int b = lane; b < nblocks; b += 32) {
        const double u = partial[(int64_t)q * nblocks + b];
        v = is_min ? fmin(v, u) : (is_max ? fmax(v, u) : v + u);
    }
    for (int o = 16; o >= 1; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_min ? fmin(v, u) : (is_max ? fmax(v, u) : v + u);
    }
    if (lane == 0) out[q] = v;
}

__global__ void catalog_weights_kernel(int64_t np, const double *w, const double *wfkp, int power, double *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        const double v = __dmul_rn(w[i], wfkp[i]);
        out[i] = power == 2 ? __dmul_rn(v, v) : v;
    }
}

// --------------------------------------------------------- interlace split
// Reference convention for the k of an index: n = i for i < N/2, i - N for
// i >= N/2 on every axis (the z Nyquist plane iz = N/2 carries k = -k_Ny).
__device__ inline int fft_index_k(int i, int n) { return i >= n / 2 ? i - n : i; }
// index of -k under that convention: -n, except the Nyquist index stays
__device__ inline int partner_k(int nk, int n) { return nk == -n / 2 ? nk : -nk; }

template <typename T>
__global__ void interlace_split_kernel(const cpx_t<T> *s1, const cpx_t<T> *s2, int n, double L, double scale,
                                       int accumulate, cpx_t<T> *herm, cpx_t<T> *anti, int64_t nh) {
    extern __shared__ double tbl[];
    AxisTable ax;
    fill_axis_table(ax, tbl, n, L, CNPC_COMP_NONE, 1);
    __syncthreads();
    const double H = L / n;
    const double inv_n3 = 1.0 / ((double)n * n * n);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += stride) {
        const Mode md = mode_of(t, n);  // FFT-order indices; recover the array indices
        const int ix = md.nx < 0 ? md.nx + n : md.nx, iy = md.ny < 0 ? md.ny + n : md.ny, iz = md.nz;
        const int nx = fft_index_k(ix, n), ny = fft_index_k(iy, n), nzk = fft_index_k(iz, n);
        // phase of k and of -k: (kx H + ky H + kz H) / 2 (mesh_generator.py:211-218)
        const double ph = 0.5 * ((ax.kx(nx) * H + ax.kx(ny) * H) + ax.kx(nzk) * H);
        const double phm = 0.5 * ((ax.kx(partner_k(nx, n)) * H + ax.kx(partner_k(ny, n)) * H) +
                                  ax.kx(partner_k(nzk, n)) * H);
        double sp, cp, sm, cm;
        sincos(ph, &sp, &cp);
        sincos(phm, &sm, &cm);
        const double a1r = (double)s1[t].x * inv_n3, a1i = (double)s1[t].y * inv_n3;
        double hr = 0.5 * a1r, hi = 0.5 * a1i, br = 0.0, bi = 0.0;
        if (s2) {
            const double a2r = (double)s2[t].x * inv_n3, a2i = (double)s2[t].y * inv_n3;
            // e1 = exp(i ph), e2 = exp(-i phm)
            const double sr = cp + cm, si = sp - sm;  // e1 + e2
            const double dr = cp - cm, di = sp + sm;  // e1 - e2
            hr += 0.25 * (a2r * sr - a2i * si);
            hi += 0.25 * (a2r * si + a2i * sr);
            const double ar = 0.25 * (a2r * dr - a2i * di), ai = 0.25 * (a2r * di + a2i * dr);
            br = ai;   // -i * A
            bi = -ar;
        } else {
            hr = a1r;
            hi = a1i;
        }
        hr *= scale, hi *= scale, br *= scale, bi *= scale;
        if (accumulate) {
            hr += (double)herm[t].x, hi += (double)herm[t].y;
            if (anti) br += (double)anti[t].x, bi += (double)anti[t].y;
        }
        herm[t] = mk<T>((T)hr, (T)hi);
        if (anti) anti[t] = mk<T>((T)br, (T)bi);
    }
}

// ------------------------------------------------------ x-space harmonics
template <typename T>
__global__ void xspace_harmonic_kernel(const T *re, const T *im, int n, double L, double bx, double by,
                                       double bz, cnpc_harmonic h, int conj, double scale, T *out_re,
                                       T *out_im) {
    extern __shared__ double xt[];  // 3 axes x n cell coordinates
    const double half = __dmul_rn(0.5, L);
    const double bc[3] = {bx, by, bz};
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        const int d = i / n, j = i % n;
        double xi = __ddiv_rn(__dmul_rn((double)j, L), (double)n);
        if (xi >= half) xi = __dsub_rn(xi, L);
        const double off = __dadd_rn(__ddiv_rn(half, (double)n), bc[d]);
        xt[i] = __dadd_rn(xi, off);
    }
    __shared__ cnpc_harmonic s_h;  // read at run-time indices by harmonic_eval
    if (threadIdx.x == 0) s_h = h;
    __syncthreads();
    const int64_t cells = (int64_t)n * n * n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += stride) {
        int iz, iy, ix;
        if (c < ((int64_t)1 << 31)) {
            uint32_t rz, ry;
            const uint32_t r = udiv31((uint32_t)c, (uint32_t)n, &rz);
            ix = (int)udiv31(r, (uint32_t)n, &ry);
            iz = (int)rz;
            iy = (int)ry;
        } else {
            iz = (int)(c % n);
            const int64_t r = c / n;
            iy = (int)(r % n);
            ix = (int)(r / n);
        }
        const double x = xt[ix], y = xt[n + iy], z = xt[2 * n + iz];
        const double rn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
        const double2 yv = harmonic_eval<double>(s_h, __ddiv_rn(x, rn), __ddiv_rn(y, rn), __ddiv_rn(z, rn), false);
        const double yr = yv.x, yi = conj ? -yv.y : yv.y;
        const double fr = (double)re[c], fi = im ? (double)im[c] : 0.0;
        out_re[c] = (T)(scale * (fr * yr - fi * yi));
        if (out_im) out_im[c] = (T)(scale * (fr * yi + fi * yr));
    }
}

// ----------------------------------------------------- survey shell sums
struct OperandDev {
    const void *p;
    const void *q;
    double scale;
    int comp;
};

template <typename T>
__device__ inline void load_operand(const OperandDev &o, int64_t t, double f, double2 *vk, double2 *vm) {
    const double s = o.scale * f;
    if (!o.p) {  // the unit spectrum
        *vk = make_double2(s, 0.0);
        *vm = *vk;
        return;
    }
    const cpx_t<T> P = static_cast<const cpx_t<T> *>(o.p)[t];
    if (!o.q) {
        *vk = make_double2(s * (double)P.x, s * (double)P.y);
        *vm = make_double2(vk->x, -vk->y);
        return;
    }
    const cpx_t<T> Q = static_cast<const cpx_t<T> *>(o.q)[t];
    // X(k) = P + i Q; X(-k) = conj(P) + i conj(Q)
    *vk = make_double2(s * ((double)P.x - (double)Q.y), s * ((double)P.y + (double)Q.x));
    *vm = make_double2(s * ((double)P.x + (double)Q.y), s * ((double)Q.x - (double)P.y));
}

// per-axis compensation tables for up to three kinds after the k table
struct CompTables {
    const double *k;
    const double *cf[4];  // indexed by kind; nullptr for CNPC_COMP_NONE
    int half;
    __device__ double factor(int kind, int nx, int ny, int nz) const {
        if (kind == CNPC_COMP_NONE) return 1.0;
        const double *c = cf[kind];
        return c[nx + half] * c[ny + half] * c[nz + half];
    }
};

__device__ inline void fill_comp_tables(CompTables &ct, double *smem, int n, double L, int p, unsigned kinds) {
    ct.half = n / 2;
    ct.k = smem;
    ct.cf[0] = nullptr;
    double *next = smem + (n + 1);
    for (int kind = 1; kind <= 3; ++kind) {
        if (kinds & (1u << kind)) {
            ct.cf[kind] = next;
            next += n + 1;
        } else {
            ct.cf[kind] = nullptr;
        }
    }
    const double H = L / n;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        const double k = kcomp(i - n / 2, L);
        smem[i] = k;
        for (int kind = 1; kind <= 3; ++kind)
            if (ct.cf[kind]) const_cast<double *>(ct.cf[kind])[i] = comp_axis(kind, p, k * H);
    }
}

template <typename T>
__global__ void survey_bins_kernel(OperandDev u, OperandDev v, int n, double L, int p, unsigned kinds,
                                   double sbr, double sbi, int has_z, cnpc_harmonic zh, int conj_z,
                                   double weight, EdgeSet edges, double *sums, BandIter bi) {
    extern __shared__ double sm[];
    CompTables ct;
    fill_comp_tables(ct, sm, n, L, p, kinds);
    const int ntab = 1 + __popc(kinds & 0xeu);
    double *bins = sm + ntab * (n + 1);
    const int nb = edges.n - 1;
    const double *e = edges_to_shared(bins + 2 * nb, edges);
    __shared__ cnpc_harmonic s_z;  // read at run-time indices by harmonic_eval
    if (threadIdx.x == 0) s_z = zh;
    for (int i = threadIdx.x; i < 2 * nb; i += blockDim.x) bins[i] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const bool sbar = sbr != 0.0 || sbi != 0.0;
    // item u = (jx, jy, iz) of the band cube folded over the signs of n_x and
    // n_y: the modes (+-jx, +-jy, iz) (one sign where jx or jy is 0 or n/2,
    // n/2 standing for -n/2) share |k| and bin; each mode keeps its own
    // operands, compensation and Z(khat), and the item sums their terms
    const int h = n / 2, R = bi.R < 0 ? h : bi.R;
    const uint32_t w1 = R + 1;
    const int64_t nq = (int64_t)w1 * w1 * w1;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < nq; base += wstride) {
        const int64_t u_ = base + lane;
        int bin = -1;
        double accr = 0.0, acci = 0.0;
        if (u_ < nq) {
            uint32_t rz, ry;
            const uint32_t r = udiv31((uint32_t)u_, w1, &rz);
            const int jx = (int)udiv31(r, w1, &ry), jy = (int)ry, iz = (int)rz;
            const double kn = knorm_from(ct.k[jx + ct.half], ct.k[jy + ct.half], ct.k[iz + ct.half]);
            bin = find_bin(kn, e, edges.n);
            if (bin >= 0) {
                const int nsx = (jx == 0 || jx == h) ? 1 : 2, nsy = (jy == 0 || jy == h) ? 1 : 2;
                const bool two = !(iz == 0 || 2 * iz == n);  // the mode -k is a distinct mode
                const double kz = ct.k[iz + ct.half];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if ((q >> 1) >= nsx || (q & 1) >= nsy) continue;
                    const int nx = ((q >> 1) || jx == h) ? -jx : jx, ny = ((q & 1) || jy == h) ? -jy : jy;
                    const int64_t tt = ((int64_t)(nx < 0 ? nx + n : nx) * n + (ny < 0 ? ny + n : ny)) * (h + 1) + iz;
                    const double kx = ct.k[nx + ct.half], ky = ct.k[ny + ct.half];
                    double2 uk, um, vk, vm;
                    load_operand<T>(u, tt, ct.factor(u.comp, nx, ny, iz), &uk, &um);
                    load_operand<T>(v, tt, ct.factor(v.comp, nx, ny, iz), &vk, &vm);
                    const double wsn = sbar ? ct.factor(CNPC_COMP_BKNOISE, nx, ny, iz) : 0.0;
                    double zr = 1.0, zi = 0.0;
                    int parity = 1;
                    if (has_z) {
                        const bool origin = kn == 0.0;
                        const double2 z = harmonic_eval<double>(s_z, origin ? 0.0 : kx / kn, origin ? 0.0 : ky / kn,
                                                                origin ? 0.0 : kz / kn, origin);
                        zr = z.x;
                        zi = conj_z ? -z.y : z.y;
                        parity = (zh.l & 1) ? -1 : 1;
                    }
                    // term(k) = (U conj V - sbar W) Z
                    double ar = uk.x * vk.x + uk.y * vk.y - sbr * wsn;
                    double ai = uk.y * vk.x - uk.x * vk.y - sbi * wsn;
                    double tr = ar * zr - ai * zi, ti = ar * zi + ai * zr;
                    if (two) {
                        ar = um.x * vm.x + um.y * vm.y - sbr * wsn;
                        ai = um.y * vm.x - um.x * vm.y - sbi * wsn;
                        tr += parity * (ar * zr - ai * zi);
                        ti += parity * (ar * zi + ai * zr);
                    }
                    accr += tr * weight;
                    acci += ti * weight;
                }
            }
        }
        double v[2] = {accr, acci};
        warp_run_add<2>(bins, nb, bin, v);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        if (bins[i] != 0.0) atomicAdd(&sums[2 * i], bins[i]);
        if (bins[nb + i] != 0.0) atomicAdd(&sums[2 * i + 1], bins[nb + i]);
    }
}

template <typename T>
__global__ void survey_source_kernel(OperandDev u, OperandDev v, int n, double L, int p, unsigned kinds,
                                     double sbr, double sbi, double band, cpx_t<T> *herm, cpx_t<T> *anti,
                                     int64_t nh) {
    extern __shared__ double sm[];
    CompTables ct;
    fill_comp_tables(ct, sm, n, L, p, kinds);
    __syncthreads();
    const bool sbar = sbr != 0.0 || sbi != 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += stride) {
        const Mode m = mode_of(t, n);
        const double kx = ct.k[m.nx + ct.half], ky = ct.k[m.ny + ct.half], kz = ct.k[m.nz + ct.half];
        const double kn = knorm_from(kx, ky, kz);
        double hr = 0.0, hi = 0.0, br = 0.0, bi = 0.0;
        if (!(band > 0.0 && kn >= band)) {
            double2 uk, um, vk, vm;
            load_operand<T>(u, t, ct.factor(u.comp, m.nx, m.ny, m.nz), &uk, &um);
            load_operand<T>(v, t, ct.factor(v.comp, m.nx, m.ny, m.nz), &vk, &vm);
            const double wsn = sbar ? ct.factor(CNPC_COMP_BKNOISE, m.nx, m.ny, m.nz) : 0.0;
            const double sr = uk.x * vk.x + uk.y * vk.y - sbr * wsn;   // src(k)
            const double si = uk.y * vk.x - uk.x * vk.y - sbi * wsn;
            const double tr = um.x * vm.x + um.y * vm.y - sbr * wsn;   // src(-k)
            const double ti = um.y * vm.x - um.x * vm.y - sbi * wsn;
            // Herm = (src(k) + conj src(-k)) / 2; B = -i (src(k) - conj src(-k)) / 2
            hr = 0.5 * (sr + tr);
            hi = 0.5 * (si - ti);
            const double dr = 0.5 * (sr - tr), di = 0.5 * (si + ti);
            br = di;
            bi = -dr;
        }
        herm[t] = mk<T>((T)hr, (T)hi);
        anti[t] = mk<T>((T)br, (T)bi);
    }
}


// out(k) += weight * (Z(k) X(k) + conj(Z(-k) X(-k))) / 2 with Z = Y(khat)
// (Y(-khat) = (-1)^l Y(khat)): the Hermitian part of Y X, accumulated.
template <typename T>
__global__ void hermitian_accumulate_kernel(OperandDev x, int n, double L, int p, unsigned kinds,
                                            cnpc_harmonic zh, double weight, cpx_t<T> *out, int64_t nh) {
    extern __shared__ double sm[];
    CompTables ct;
    fill_comp_tables(ct, sm, n, L, p, kinds);
    __shared__ cnpc_harmonic s_z;  // read at run-time indices by harmonic_eval
    if (threadIdx.x == 0) s_z = zh;
    __syncthreads();
    const int parity = (zh.l & 1) ? -1 : 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += stride) {
        const Mode m = mode_of(t, n);
        const double kx = ct.k[m.nx + ct.half], ky = ct.k[m.ny + ct.half], kz = ct.k[m.nz + ct.half];
        const double kn = knorm_from(kx, ky, kz);
        const bool origin = kn == 0.0;
        const double2 y = harmonic_eval<double>(s_z, origin ? 0.0 : kx / kn, origin ? 0.0 : ky / kn,
                                                origin ? 0.0 : kz / kn, origin);
        double2 xk, xm;
        load_operand<T>(x, t, ct.factor(x.comp, m.nx, m.ny, m.nz), &xk, &xm);
        // Z(k) X(k)
        const double ar = y.x * xk.x - y.y * xk.y, ai = y.x * xk.y + y.y * xk.x;
        // conj(Z(-k) X(-k)) = parity * conj(Y) conj(X(-k))
        const double br = parity * (y.x * xm.x - y.y * xm.y);
        const double bi = -parity * (y.x * xm.y + y.y * xm.x);
        const double hr = 0.5 * weight * (ar + br), hi = 0.5 * weight * (ai + bi);
        out[t] = mk<T>((T)((double)out[t].x + hr), (T)((double)out[t].y + hi));
    }
}

// --------------------------------------------------- x-space reductions
template <typename T>
__global__ void product_sum_kernel(int64_t ncell, int nf, const T *r0, const T *i0, const T *r1, const T *i1,
                                   const T *r2, const T *i2, double *partial) {
    double sr = 0.0, si = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += stride) {
        double pr = (double)r0[c], pi = i0 ? (double)i0[c] : 0.0;
        if (nf > 1) {
            const double ar = (double)r1[c], ai = i1 ? (double)i1[c] : 0.0;
            const double tr = pr * ar - pi * ai;
            pi = pr * ai + pi * ar;
            pr = tr;
        }
        if (nf > 2) {
            const double ar = (double)r2[c], ai = i2 ? (double)i2[c] : 0.0;
            const double tr = pr * ar - pi * ai;
            pi = pr * ai + pi * ar;
            pr = tr;
        }
        sr += pr;
        si += pi;
    }
    __shared__ double red[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o >= 1; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) red[0][warp] = sr, red[1][warp] = si;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) a += red[0][i], b += red[1][i];
        partial[blockIdx.x] = a;
        partial[gridDim.x + blockIdx.x] = b;
    }
}

template <typename T>
__global__ void axpby_kernel(int64_t ncell, double a, const T *x, double b, const T *y, T *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += stride) {
        double v = __dmul_rn(a, (double)x[c]);
        if (y) v = __dadd_rn(v, __dmul_rn(b, (double)y[c]));
        out[c] = (T)v;
    }
}

static int check_operand(cnpc_ctx *ctx, const cnpc_operand *o, OperandDev *d) {
    CNPC_REQUIRE(ctx, o != nullptr, "null operand");
    CNPC_REQUIRE(ctx, o->p != nullptr || o->q == nullptr, "operand with q but no p");
    CNPC_REQUIRE(ctx, o->comp >= CNPC_COMP_NONE && o->comp <= CNPC_COMP_BKNOISE, "bad compensation kind");
    d->p = o->p;
    d->q = o->q;
    d->scale = o->scale;
    d->comp = o->comp;
    return CNPC_OK;
}

}  // namespace cnpc

using namespace cnpc;

extern "C" {

int cnpc_catalog_decode(cnpc_ctx *ctx, const void *d_rows, int64_t nrows, const cnpc_catalog_spec *h_spec,
                        double *d_pos, double *d_weight, double *d_wfkp, double *d_nz, int64_t *h_kept,
                        cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, h_spec != nullptr && h_kept != nullptr, "null argument");
    CNPC_REQUIRE(ctx, nrows >= 0, "negative row count");
    CNPC_REQUIRE(ctx, nrows == 0 || (d_rows && d_pos && d_weight && d_wfkp && d_nz), "null buffer");
    CNPC_REQUIRE(ctx, h_spec->row_bytes > 0 || nrows == 0, "row_bytes must be positive");
    const cnpc_catalog_spec &sp = *h_spec;
    for (int c = 0; c < CNPC_NCOLS; ++c) {
        const cnpc_column &col = sp.col[c];
        CNPC_REQUIRE(ctx, col.type >= CNPC_CT_ABSENT && col.type <= CNPC_CT_BOOL, "bad column type");
        if (col.type != CNPC_CT_ABSENT) CNPC_REQUIRE(ctx, col.offset >= 0, "negative column offset");
    }
    const int need[] = {CNPC_COL_RA, CNPC_COL_DEC, CNPC_COL_Z, CNPC_COL_FKP};
    for (int c : need) CNPC_REQUIRE(ctx, sp.col[c].type != CNPC_CT_ABSENT, "RA, DEC, Z and WEIGHT_FKP are required");
    CNPC_REQUIRE(ctx, sp.weight_rule >= CNPC_W_COLUMN && sp.weight_rule <= CNPC_W_EBOSS, "bad weight rule");
    if (sp.weight_rule == CNPC_W_COLUMN)
        CNPC_REQUIRE(ctx, sp.col[CNPC_COL_WEIGHT].type != CNPC_CT_ABSENT, "weight column missing");
    if (sp.weight_rule == CNPC_W_BOSS || sp.weight_rule == CNPC_W_EBOSS)
        CNPC_REQUIRE(ctx, sp.col[CNPC_COL_SYSTOT].type && sp.col[CNPC_COL_NOZ].type && sp.col[CNPC_COL_CP].type,
                     "completeness columns missing");
    CNPC_REQUIRE(ctx, sp.cosmology == CNPC_COSMO_FLAT_LCDM || sp.cosmology == CNPC_COSMO_PLANCK18,
                 "bad cosmology model");
    CNPC_REQUIRE(ctx, sp.h > 0.0 && (sp.cosmology == CNPC_COSMO_PLANCK18 || (sp.omega_m > 0.0 && sp.omega_m < 1.0)),
                 "cosmology out of range");
    *h_kept = 0;
    if (nrows == 0) return CNPC_OK;
    for (int c = 0; c < CNPC_NCOLS; ++c) {
        const cnpc_column &col = sp.col[c];
        if (col.type == CNPC_CT_ABSENT) continue;
        const int nb = (col.type == CNPC_CT_F64 || col.type == CNPC_CT_I64) ? 8
                       : (col.type == CNPC_CT_F32 || col.type == CNPC_CT_I32) ? 4
                       : (col.type == CNPC_CT_I16) ? 2 : 1;
        CNPC_REQUIRE(ctx, col.offset + nb <= sp.row_bytes, "column extends past the row");
    }
    CatalogParams p;
    p.row_bytes = sp.row_bytes;
    std::memcpy(p.col, sp.col, sizeof(p.col));
    p.weight_rule = sp.weight_rule;
    p.has_zrange = sp.has_zrange;
    p.z_min = sp.z_min;
    p.z_max = sp.z_max;
    p.omega_m = sp.omega_m;
    p.h = sp.h;
    p.hubble_distance = 299792.458 / (100.0 * sp.h);
    p.planck18 = sp.cosmology == CNPC_COSMO_PLANCK18;
    p.ogamma0 = p.ode0 = p.nu_prefac = p.nu_y = p.nu_massless = 0.0;
    if (p.planck18) {
        const Planck18Radiation r = planck18_radiation();
        p.omega_m = 0.30966;
        p.ogamma0 = r.ogamma0;
        p.ode0 = r.ode0;
        p.nu_prefac = r.nu_prefac;
        p.nu_y = r.nu_y;
        p.nu_massless = r.nu_massless;
        p.hubble_distance = r.hubble_distance;
    }
    p.gl = gauss_legendre16();
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nblk64 = (nrows + kRowsPerBlock - 1) / kRowsPerBlock;
    CNPC_REQUIRE(ctx, nblk64 < (1 << 30), "too many rows");
    const int nblk = (int)nblk64;
    const size_t bytes = sizeof(int) * nblk + 256 + sizeof(long long) * (nblk + 1);
    int st = ensure_buffer(ctx, &ctx->aux, &ctx->aux_bytes, bytes, s);
    if (st) return st;
    int *counts = static_cast<int *>(ctx->aux);
    long long *offsets = reinterpret_cast<long long *>(static_cast<char *>(ctx->aux) +
                                                       ((sizeof(int) * nblk + 255) / 256 * 256));
    const uint8_t *rows = static_cast<const uint8_t *>(d_rows);
    catalog_count_kernel<<<nblk, 256, 0, s>>>(rows, nrows, p, counts);
    block_scan_kernel<<<1, 1024, 0, s>>>(counts, nblk, offsets);
    catalog_decode_kernel<<<nblk, 256, 0, s>>>(rows, nrows, p, offsets, d_pos, d_weight, d_wfkp, d_nz);
    st = check_launch(ctx, "catalog_decode");
    if (st) return st;
    long long kept = 0;
    st = check_cuda(ctx, cudaMemcpyAsync(&kept, offsets + nblk, sizeof(long long), cudaMemcpyDeviceToHost, s),
                    "copy row count");
    if (st) return st;
    st = check_cuda(ctx, cudaStreamSynchronize(s), "catalog_decode sync");
    if (st) return st;
    *h_kept = kept;
    return CNPC_OK;
}

int cnpc_particle_sums(cnpc_ctx *ctx, int64_t np, const double *d_pos, const double *d_weight,
                       const double *d_wfkp, const double *d_nz, const cnpc_harmonic *h_ylm, int nharm,
                       double *d_out, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, np >= 0, "negative particle count");
    CNPC_REQUIRE(ctx, d_out != nullptr, "null output");
    CNPC_REQUIRE(ctx, np == 0 || (d_pos && d_weight && d_wfkp && d_nz), "null buffer");
    CNPC_REQUIRE(ctx, nharm >= 0 && nharm <= CNPC_MAX_HARMONICS, "nharm out of range");
    CNPC_REQUIRE(ctx, nharm == 0 || h_ylm != nullptr, "null harmonic table");
    YlmSet ys;
    ys.n = nharm;
    for (int i = 0; i < nharm; ++i) {
        CNPC_REQUIRE(ctx, h_ylm[i].l >= 0 && h_ylm[i].l <= 8, "harmonic degree out of range");
        ys.h[i] = h_ylm[i];
    }
    const int nsum = CNPC_PSUM_COUNT + 2 * nharm;
    const int nq = nsum + 6;
    cudaStream_t s = (cudaStream_t)stream;
    int st = ensure_buffer(ctx, &ctx->aux, &ctx->aux_bytes, sizeof(double) * nq * kPsumBlocks, s);
    if (st) return st;
    double *partial = static_cast<double *>(ctx->aux);
    particle_sums_kernel<<<kPsumBlocks, kPsumThreads, 0, s>>>(np, d_pos, d_weight, d_wfkp, d_nz, ys, partial);
    partials_reduce_kernel<<<(nq + 7) / 8, 256, 0, s>>>(partial, kPsumBlocks, nsum, 6, d_out);
    return check_launch(ctx, "particle_sums");
}

int cnpc_catalog_weights(cnpc_ctx *ctx, int64_t np, const double *d_weight, const double *d_wfkp, int power,
                         double *d_out, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, power == 1 || power == 2, "power must be 1 or 2");
    CNPC_REQUIRE(ctx, np >= 0, "negative particle count");
    if (np == 0) return CNPC_OK;
    CNPC_REQUIRE(ctx, d_weight && d_wfkp && d_out, "null buffer");
    catalog_weights_kernel<<<grid_for(ctx, np, 256), 256, 0, (cudaStream_t)stream>>>(np, d_weight, d_wfkp, power,
                                                                                    d_out);
    return check_launch(ctx, "catalog_weights");
}

int cnpc_interlace_split(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec,
                         const void *d_spec2, double scale, int accumulate, void *d_herm, void *d_anti,
                         cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, d_spec && d_herm, "null buffer");
    CNPC_REQUIRE(ctx, d_spec2 == nullptr || d_anti != nullptr, "interlaced split needs d_anti");
    const int64_t nh = half_modes(n);
    const int threads = 256;
    const size_t smem = sizeof(double) * (n + 1);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == CNPC_F32)
        interlace_split_kernel<float><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            (const float2 *)d_spec, (const float2 *)d_spec2, n, boxsize, scale, accumulate, (float2 *)d_herm,
            (float2 *)d_anti, nh);
    else
        interlace_split_kernel<double><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            (const double2 *)d_spec, (const double2 *)d_spec2, n, boxsize, scale, accumulate,
            (double2 *)d_herm, (double2 *)d_anti, nh);
    return check_launch(ctx, "interlace_split_kernel");
}

int cnpc_xspace_harmonic(cnpc_ctx *ctx, int dtype, int n, double boxsize, const double *h_boxcenter,
                         const void *d_re, const void *d_im, const cnpc_harmonic *h_y, int conj, double scale,
                         void *d_out_re, void *d_out_im, cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, h_boxcenter && h_y && d_re && d_out_re, "null argument");
    CNPC_REQUIRE(ctx, h_y->l >= 0 && h_y->l <= 8 && std::abs(h_y->m) <= h_y->l, "harmonic out of range");
    const int64_t cells = (int64_t)n * n * n;
    const int threads = 256;
    const size_t smem = sizeof(double) * 3 * n;
    cudaStream_t s = (cudaStream_t)stream;
    if (smem > 48 * 1024) {
        const cudaError_t e = dtype == CNPC_F32
            ? cudaFuncSetAttribute(xspace_harmonic_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
            : cudaFuncSetAttribute(xspace_harmonic_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        st = check_cuda(ctx, e, "xspace smem");
        if (st) return st;
    }
    if (dtype == CNPC_F32)
        xspace_harmonic_kernel<float><<<grid_for(ctx, cells, threads), threads, smem, s>>>(
            (const float *)d_re, (const float *)d_im, n, boxsize, h_boxcenter[0], h_boxcenter[1], h_boxcenter[2],
            *h_y, conj, scale, (float *)d_out_re, (float *)d_out_im);
    else
        xspace_harmonic_kernel<double><<<grid_for(ctx, cells, threads), threads, smem, s>>>(
            (const double *)d_re, (const double *)d_im, n, boxsize, h_boxcenter[0], h_boxcenter[1], h_boxcenter[2],
            *h_y, conj, scale, (double *)d_out_re, (double *)d_out_im);
    return check_launch(ctx, "xspace_harmonic_kernel");
}

int cnpc_survey_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, int window, const cnpc_operand *u,
                     const cnpc_operand *v, double sbar_re, double sbar_im, const cnpc_harmonic *h_z,
                     int conj_z, double weight, const double *h_edges, int nedges, double *d_sums,
                     cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, window >= 1 && window <= 4, "window must be 1..4");
    CNPC_REQUIRE(ctx, d_sums != nullptr, "null output");
    OperandDev du, dv;
    if ((st = check_operand(ctx, u, &du))) return st;
    if ((st = check_operand(ctx, v, &dv))) return st;
    if (h_z) CNPC_REQUIRE(ctx, h_z->l >= 0 && h_z->l <= 8 && std::abs(h_z->m) <= h_z->l, "harmonic out of range");
    EdgeSet es;
    if ((st = load_edges(ctx, h_edges, nedges, &es))) return st;
    cnpc_harmonic zh{};
    if (h_z) zh = *h_z;
    unsigned kinds = (1u << du.comp) | (1u << dv.comp);
    if (sbar_re != 0.0 || sbar_im != 0.0) kinds |= 1u << CNPC_COMP_BKNOISE;
    kinds &= 0xeu;
    const int ntab = 1 + __builtin_popcount(kinds);
    const int nb = nedges - 1;
    cudaStream_t s = (cudaStream_t)stream;
    st = check_cuda(ctx, cudaMemsetAsync(d_sums, 0, sizeof(double) * 2 * nb, s), "memset");
    if (st) return st;
    const BandIter bi = band_iter(n, boxsize, h_edges[nedges - 1]);
    const int64_t rq = bi.R < 0 ? n / 2 : bi.R;
    const int64_t nh = (rq + 1) * (rq + 1) * (rq + 1);  // sign-folded items
    const int threads = 256;
    const size_t smem = sizeof(double) * (ntab * (n + 1) + 2 * nb + nedges);
    if (dtype == CNPC_F32)
        survey_bins_kernel<float><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            du, dv, n, boxsize, window, kinds, sbar_re, sbar_im, h_z ? 1 : 0, zh, conj_z, weight, es, d_sums, bi);
    else
        survey_bins_kernel<double><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            du, dv, n, boxsize, window, kinds, sbar_re, sbar_im, h_z ? 1 : 0, zh, conj_z, weight, es, d_sums, bi);
    return check_launch(ctx, "survey_bins_kernel");
}

int cnpc_survey_source(cnpc_ctx *ctx, int dtype, int n, double boxsize, int window, const cnpc_operand *u,
                       const cnpc_operand *v, double sbar_re, double sbar_im, double band_kmax, void *d_herm,
                       void *d_anti, cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, window >= 1 && window <= 4, "window must be 1..4");
    CNPC_REQUIRE(ctx, d_herm && d_anti, "null output");
    OperandDev du, dv;
    if ((st = check_operand(ctx, u, &du))) return st;
    if ((st = check_operand(ctx, v, &dv))) return st;
    unsigned kinds = (1u << du.comp) | (1u << dv.comp);
    if (sbar_re != 0.0 || sbar_im != 0.0) kinds |= 1u << CNPC_COMP_BKNOISE;
    kinds &= 0xeu;
    const int ntab = 1 + __builtin_popcount(kinds);
    const int64_t nh = half_modes(n);
    const int threads = 256;
    const size_t smem = sizeof(double) * ntab * (n + 1);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == CNPC_F32)
        survey_source_kernel<float><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            du, dv, n, boxsize, window, kinds, sbar_re, sbar_im, band_kmax, (float2 *)d_herm, (float2 *)d_anti, nh);
    else
        survey_source_kernel<double><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            du, dv, n, boxsize, window, kinds, sbar_re, sbar_im, band_kmax, (double2 *)d_herm, (double2 *)d_anti, nh);
    return check_launch(ctx, "survey_source_kernel");
}

int cnpc_survey_hermitian_accumulate(cnpc_ctx *ctx, int dtype, int n, double boxsize, int window,
                                     const cnpc_operand *x, const cnpc_harmonic *h_y, double weight,
                                     void *d_out, cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, window >= 1 && window <= 4, "window must be 1..4");
    CNPC_REQUIRE(ctx, h_y && d_out, "null argument");
    CNPC_REQUIRE(ctx, h_y->l >= 0 && h_y->l <= 8 && std::abs(h_y->m) <= h_y->l, "harmonic out of range");
    OperandDev dx;
    if ((st = check_operand(ctx, x, &dx))) return st;
    const unsigned kinds = (1u << dx.comp) & 0xeu;
    const int ntab = 1 + __builtin_popcount(kinds);
    const int64_t nh = half_modes(n);
    const int threads = 256;
    const size_t smem = sizeof(double) * ntab * (n + 1);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == CNPC_F32)
        hermitian_accumulate_kernel<float><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            dx, n, boxsize, window, kinds, *h_y, weight, (float2 *)d_out, nh);
    else
        hermitian_accumulate_kernel<double><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            dx, n, boxsize, window, kinds, *h_y, weight, (double2 *)d_out, nh);
    return check_launch(ctx, "hermitian_accumulate_kernel");
}

int cnpc_field_product_sum(cnpc_ctx *ctx, int dtype, int64_t ncell, int nf, const void *const *h_re,
                           const void *const *h_im, double *d_out, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    CNPC_REQUIRE(ctx, nf >= 1 && nf <= 3, "nf must be 1..3");
    CNPC_REQUIRE(ctx, ncell > 0 && h_re && d_out, "null argument");
    const void *r[3] = {nullptr, nullptr, nullptr}, *im[3] = {nullptr, nullptr, nullptr};
    for (int i = 0; i < nf; ++i) {
        CNPC_REQUIRE(ctx, h_re[i] != nullptr, "null field");
        r[i] = h_re[i];
        im[i] = h_im ? h_im[i] : nullptr;
    }
    const int nblocks = ctx->num_sms * 4;
    cudaStream_t s = (cudaStream_t)stream;
    int st = ensure_buffer(ctx, &ctx->aux, &ctx->aux_bytes, sizeof(double) * 2 * nblocks, s);
    if (st) return st;
    double *partial = static_cast<double *>(ctx->aux);
    if (dtype == CNPC_F32)
        product_sum_kernel<float><<<nblocks, 256, 0, s>>>(ncell, nf, (const float *)r[0], (const float *)im[0],
                                                          (const float *)r[1], (const float *)im[1],
                                                          (const float *)r[2], (const float *)im[2], partial);
    else
        product_sum_kernel<double><<<nblocks, 256, 0, s>>>(ncell, nf, (const double *)r[0], (const double *)im[0],
                                                           (const double *)r[1], (const double *)im[1],
                                                           (const double *)r[2], (const double *)im[2], partial);
    partials_reduce_kernel<<<1, 64, 0, s>>>(partial, nblocks, 2, 0, d_out);
    return check_launch(ctx, "product_sum_kernel");
}

int cnpc_field_axpby(cnpc_ctx *ctx, int dtype, int64_t ncell, double a, const void *d_x, double b,
                     const void *d_y, void *d_out, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    CNPC_REQUIRE(ctx, ncell > 0 && d_x && d_out, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == CNPC_F32)
        axpby_kernel<float><<<grid_for(ctx, ncell, 256), 256, 0, s>>>(ncell, a, (const float *)d_x, b,
                                                                      (const float *)d_y, (float *)d_out);
    else
        axpby_kernel<double><<<grid_for(ctx, ncell, 256), 256, 0, s>>>(ncell, a, (const double *)d_x, b,
                                                                       (const double *)d_y, (double *)d_out);
    return check_launch(ctx, "axpby_kernel");
}

}  // extern "C"
