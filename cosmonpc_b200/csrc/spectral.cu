// k-space stages: forward finish (interlace + compensation), mode counts,
// shell sums for pk and the bk shot-noise terms, and shell-spectrum synthesis.
#include <cmath>
#include <cstring>

#include "bins.cuh"

namespace cnpc {

// ---------------------------------------------------------------- forward
template <typename T>
__global__ void forward_finish_kernel(cpx_t<T> *spec, const cpx_t<T> *spec2, int n, double L,
                                      double inv_n3, double scale, int comp, int p, double k0,
                                      double band, cpx_t<T> *band_out, double band_out_k, int64_t nq) {
    extern __shared__ double tbl[];
    AxisTable ax;
    fill_axis_table(ax, tbl, n, L, comp, p);
    const double H = L / n;
    // the interlacing phase e^{i (kx + ky + kz) H / 2} as the product of one
    // factor per axis, each from a per-block table of e^{i k H / 2}
    double2 *ph = reinterpret_cast<double2 *>(tbl + 2 * (n + 1));  // [n + 1]
    if (spec2)
        for (int i = threadIdx.x; i <= n; i += blockDim.x) {
            double sp, cp;
            sincos(0.5 * (ax.k[i] * H), &sp, &cp);
            ph[i] = make_double2(cp, sp);
        }
    __syncthreads();
    // item u = (jx, jy, iz), jx, jy, iz in [0, n/2]: the 1-4 modes
    // (+-jx, +-jy, iz) (one sign where jx or jy is 0 or n/2, n/2 standing for
    // -n/2) share |k| and so the band tests; their loads are issued together
    const int h = n / 2;
    const uint32_t w1 = h + 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nq; u += stride) {
        uint32_t rz, ry;
        const uint32_t r = udiv31((uint32_t)u, w1, &rz);
        const int jx = (int)udiv31(r, w1, &ry), jy = (int)ry, iz = (int)rz;
        const double kn = knorm_from(ax.kx(jx), ax.kx(jy), ax.kx(iz));
        const bool cut = band > 0.0 && kn >= band;
        const bool in_out = kn < band_out_k;
        const int nsx = (jx == 0 || jx == h) ? 1 : 2, nsy = (jy == 0 || jy == h) ? 1 : 2;
        // mode q = 2 sx + sy of the orbit, present when sx < nsx and sy < nsy
        auto mode_nx = [&](int q) { return ((q >> 1) || jx == h) ? -jx : jx; };
        auto mode_ny = [&](int q) { return ((q & 1) || jy == h) ? -jy : jy; };
        auto mode_t = [&](int q) {
            const int nx = mode_nx(q), ny = mode_ny(q);
            return ((int64_t)(nx < 0 ? nx + n : nx) * n + (ny < 0 ? ny + n : ny)) * w1 + iz;
        };
        cpx_t<T> va[4], vb[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if ((q >> 1) < nsx && (q & 1) < nsy) {
                va[q] = spec[mode_t(q)];
                if (spec2) vb[q] = spec2[mode_t(q)];
            }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if ((q >> 1) >= nsx || (q & 1) >= nsy) continue;
            const int64_t t = mode_t(q);
            const int mxq = mode_nx(q), myq = mode_ny(q);
            double re = (double)va[q].x * inv_n3, im = (double)va[q].y * inv_n3;
            if (spec2) {
                const double2 ex = ph[mxq + h], ey = ph[myq + h], ez = ph[iz + h];
                const double cxy = ex.x * ey.x - ex.y * ey.y, sxy = ex.x * ey.y + ex.y * ey.x;
                const double cp = cxy * ez.x - sxy * ez.y, sp = cxy * ez.y + sxy * ez.x;
                const double r2 = (double)vb[q].x * inv_n3, i2 = (double)vb[q].y * inv_n3;
                re = 0.5 * re + 0.5 * (r2 * cp - i2 * sp);
                im = 0.5 * im + 0.5 * (r2 * sp + i2 * cp);
            }
            double f = scale;
            if (ax.cf) f *= ax.f(mxq) * ax.f(myq) * ax.f(iz);
            re *= f;
            im *= f;
            if (t == 0 && !isnan(k0)) {
                re = k0;
                im = 0.0;
            }
            if (cut) re = im = 0.0;
            spec[t] = mk<T>((T)re, (T)im);
            // band_out may be spec2: this thread read its element t above
            if (band_out) band_out[t] = in_out ? mk<T>((T)re, (T)im) : mk<T>((T)0, (T)0);
        }
    }
}

// ------------------------------------------------------------ mode counts
// The counts fold the half spectrum over the signs of n_x and n_y: k = 2 n pi / L
// is odd in n bit for bit and |k| squares it, so the modes (+-n_x, +-n_y, n_z)
// share |k| and bin.  The quadrant n_x, n_y in [0, R] (R = n/2 on the whole
// spectrum, where n_d = n/2 stands for the single mode -n/2) is summed with
// weight 2 per axis for 0 < n_d < n/2 and 1 otherwise, times the Hermitian
// multiplicity of n_z: the same counts (exact integers) and |k| sums to
// rounding, over a quarter of the modes.  Consecutive u are consecutive n_z
// of one row, as warp_run_add wants.
struct QuadIter {
    int n, R, RZ;  // n_x, n_y in [0, R], n_z in [0, RZ]
    int64_t count;
};

inline QuadIter quad_iter(int n, double boxsize, double e_last) {
    const BandIter bi = band_iter(n, boxsize, e_last);
    QuadIter q;
    q.n = n;
    q.R = bi.R < 0 ? n / 2 : bi.R;
    q.RZ = bi.R < 0 ? n / 2 : bi.R;
    q.count = (int64_t)(q.R + 1) * (q.R + 1) * (q.RZ + 1);
    return q;
}

__global__ void kbin_counts_kernel(int n, double L, EdgeSet edges, double *counts, double *ksum, QuadIter qi) {
    extern __shared__ double sm[];
    AxisTable ax;
    fill_axis_table(ax, sm, n, L, CNPC_COMP_NONE, 1);
    double *bins = sm + (n + 1);
    const int nb = edges.n - 1;
    const double *e = edges_to_shared(bins + 2 * nb, edges);
    for (int i = threadIdx.x; i < 2 * nb; i += blockDim.x) bins[i] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    const uint32_t w = qi.R + 1, nzc = qi.RZ + 1;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < qi.count;
         base += wstride) {
        const int64_t t = base + lane;
        int bin = -1;
        double kn = 0.0, mult = 0.0;
        if (t < qi.count) {
            int iz, jy, jx;
            if (t < ((int64_t)1 << 31)) {
                uint32_t rz, ry;
                const uint32_t r = udiv31((uint32_t)t, nzc, &rz);
                jx = (int)udiv31(r, w, &ry);
                iz = (int)rz;
                jy = (int)ry;
            } else {
                iz = (int)(t % nzc);
                const int64_t r = t / nzc;
                jy = (int)(r % w);
                jx = (int)(r / w);
            }
            kn = knorm_from(ax.kx(jx), ax.kx(jy), ax.kx(iz));
            bin = find_bin(kn, e, edges.n);
            const int wx = (jx == 0 || 2 * jx == n) ? 1 : 2, wy = (jy == 0 || 2 * jy == n) ? 1 : 2;
            const int wz = (iz == 0 || 2 * iz == n) ? 1 : 2;
            mult = (double)(wx * wy * wz);
        }
        double v[2] = {mult, mult * kn};
        warp_run_add<2>(bins, nb, bin, v);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        if (bins[i] != 0.0) atomicAdd(&counts[i], bins[i]);
        if (bins[nb + i] != 0.0) atomicAdd(&ksum[i], bins[nb + i]);
    }
}

// --------------------------------------------------------------- pk sums
struct PoleSet {
    int n;
    int l[CNPC_MAX_POLES];
    double los[3];
};

template <typename T>
__global__ void pk_bins_kernel(const cpx_t<T> *a, const cpx_t<T> *b, int n, double L, EdgeSet edges,
                               PoleSet poles, double *sums, BandIter bi) {
    extern __shared__ double sm[];
    AxisTable ax;
    fill_axis_table(ax, sm, n, L, CNPC_COMP_NONE, 1);
    double *bins = sm + (n + 1);
    const int nb = edges.n - 1;
    const double *e = edges_to_shared(bins + poles.n * nb, edges);
    for (int i = threadIdx.x; i < poles.n * nb; i += blockDim.x) bins[i] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    // item u = (jx, jy, iz) of the band cube folded over the signs of n_x and
    // n_y: the modes (+-jx, +-jy, iz) (one sign where jx or jy is 0 or n/2,
    // n/2 standing for -n/2) share |k| and bin, and with the line of sight
    // along z also mu and the Legendre values, which then run once per item
    const bool los_z = poles.los[0] == 0.0 && poles.los[1] == 0.0;
    const int h = n / 2, R = bi.R < 0 ? h : bi.R;
    const uint32_t w1 = R + 1;
    const int64_t nq = (int64_t)w1 * w1 * w1;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < nq;
         base += wstride) {
        const int64_t u = base + lane;
        int bin = -1;
        int jx = 0, jy = 0, iz = 0, nsx = 1, nsy = 1;
        double kn = 0.0, mult = 0.0;
        if (u < nq) {
            uint32_t rz, ry;
            const uint32_t r = udiv31((uint32_t)u, w1, &rz);
            jx = (int)udiv31(r, w1, &ry);
            jy = (int)ry;
            iz = (int)rz;
            kn = knorm_from(ax.kx(jx), ax.kx(jy), ax.kx(iz));
            bin = find_bin(kn, e, edges.n);
            nsx = (jx == 0 || jx == h) ? 1 : 2;
            nsy = (jy == 0 || jy == h) ? 1 : 2;
            mult = (iz == 0 || 2 * iz == n) ? 1.0 : 2.0;
        }
        // the orbit's members: power |delta|^2 and mu of member q = 2 sx + sy
        double pvq[4] = {0.0, 0.0, 0.0, 0.0}, muq[4] = {0.0, 0.0, 0.0, 0.0};
        if (bin >= 0) {
            const double kz = ax.kx(iz);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if ((q >> 1) >= nsx || (q & 1) >= nsy) continue;
                const int nx = ((q >> 1) || jx == h) ? -jx : jx, ny = ((q & 1) || jy == h) ? -jy : jy;
                const int64_t tt = ((int64_t)(nx < 0 ? nx + n : nx) * n + (ny < 0 ? ny + n : ny)) * (h + 1) + iz;
                const cpx_t<T> va = a[tt], vb = b[tt];
                pvq[q] = mult * ((double)va.x * (double)vb.x + (double)va.y * (double)vb.y);
                if (kn > 0.0)
                    muq[q] = (ax.kx(nx) / kn) * poles.los[0] + (ax.kx(ny) / kn) * poles.los[1] +
                             (kz / kn) * poles.los[2];
            }
        }
        // poles in groups of four (a warp-uniform loop)
        for (int q0 = 0; q0 < poles.n; q0 += 4) {
            const int np_ = poles.n - q0 < 4 ? poles.n - q0 : 4;
            double v[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (c >= np_) break;
                const int l = poles.l[q0 + c];
                v[c] = 0.0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (los_z && q > 0) break;  // one mu for the orbit
                    // Legendre P_l(mu) by the three-term recurrence
                    const double mu = muq[q];
                    double p0 = 1.0, p1 = mu;
                    double pl = (l == 0) ? 1.0 : mu;
                    for (int j = 1; j < l; ++j) {
                        pl = ((2 * j + 1) * mu * p1 - j * p0) / (j + 1);
                        p0 = p1;
                        p1 = pl;
                    }
                    if (los_z)
                        v[c] += ((pvq[0] + pvq[1]) + (pvq[2] + pvq[3])) * pl;
                    else
                        v[c] += pvq[q] * pl;
                }
            }
            warp_run_add<4>(bins + q0 * nb, nb, bin, v, np_);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < poles.n * nb; i += blockDim.x)
        if (bins[i] != 0.0) atomicAdd(&sums[i], bins[i]);
}

// ------------------------------------------------------- shot-noise sums
// Up to kSnMaxCfg shot-noise configurations share one pass over the modes
// (the decode, |k|, bin and spectrum loads); each has its own sn0, Y_L0,
// sums and source.
constexpr int kSnMaxCfg = 2;
struct SnCfg {
    double sn0[kSnMaxCfg];
    int use_y[kSnMaxCfg];
    cnpc_harmonic yl0[kSnMaxCfg];
    double *sums[kSnMaxCfg];
    void *source[kSnMaxCfg];
};

template <typename T, int NC>
__global__ void sn_bins_kernel(const cpx_t<T> *a, const cpx_t<T> *b, int n, double L, double vsq, int p,
                               EdgeSet edges, const SnCfg cfg, double band, int64_t nq) {
    extern __shared__ double sm[];
    bool any_sn0 = false, any_src = false;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        any_sn0 |= cfg.sn0[c] != 0.0;
        any_src |= cfg.source[c] != nullptr;
    }
    AxisTable ax;
    fill_axis_table(ax, sm, n, L, any_sn0 ? CNPC_COMP_BKNOISE : CNPC_COMP_NONE, p);
    // per configuration nb + 1 bins: the shell sums, then the full-space sum of
    // its source (the source's x = 0 value)
    double *bins = sm + 2 * (n + 1);
    const int nb = edges.n - 1, nbt = nb + 1;
    const double *e = edges_to_shared(bins + NC * nbt, edges);
    __shared__ cnpc_harmonic s_y[NC];  // read at run-time indices by harmonic_eval
    if (threadIdx.x < NC) s_y[threadIdx.x] = cfg.yl0[threadIdx.x];
    for (int i = threadIdx.x; i < NC * nbt; i += blockDim.x) bins[i] = 0.0;
    __syncthreads();
    double tot[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) tot[c] = 0.0;
    const int lane = threadIdx.x & 31;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    const int h = n / 2;
    const uint32_t w1 = h + 1;
    // item u = (jx, jy, iz), jx, jy, iz in [0, n/2]: the modes (+-jx, +-jy, iz)
    // (one sign where jx or jy is 0 or n/2, n/2 standing for -n/2) share |k|,
    // bin and Y_L0 (a function of k_z / |k|); their values are summed in the
    // item before the warp's run sums
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < nq;
         base += wstride) {
        const int64_t u = base + lane;
        int bin = -1;
        double val[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) val[c] = 0.0;
        if (u < nq) {
            uint32_t rz, ry;
            const uint32_t r = udiv31((uint32_t)u, w1, &rz);
            const int jx = (int)udiv31(r, w1, &ry), jy = (int)ry, iz = (int)rz;
            const double kx = ax.kx(jx), ky = ax.kx(jy), kz = ax.kx(iz);
            const double kn = knorm_from(kx, ky, kz);
            bin = find_bin(kn, e, edges.n);
            const bool keep = !(band > 0.0) || kn < band;
            const double mult = (iz == 0 || 2 * iz == n) ? 1.0 : 2.0;
            const int nsx = (jx == 0 || jx == h) ? 1 : 2, nsy = (jy == 0 || jy == h) ? 1 : 2;
            const bool live = bin >= 0 || (any_src && keep);
            double y[NC];
            if (live && bin >= 0) {
                const bool origin = kn == 0.0;
                const double ik = origin ? 0.0 : 1.0 / kn;
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    y[c] = cfg.use_y[c] ? harmonic_eval<double>(s_y[c], kx * ik, ky * ik, kz * ik, origin).x : 1.0;
            }
            for (int sx = 0; sx < nsx; ++sx)
                for (int sy = 0; sy < nsy; ++sy) {
                    const int nx = (sx || jx == h) ? -jx : jx, ny = (sy || jy == h) ? -jy : jy;
                    const int ix = nx < 0 ? nx + n : nx, iy = ny < 0 ? ny + n : ny;
                    const int64_t t = ((int64_t)ix * n + iy) * w1 + iz;
                    if (live) {
                        const cpx_t<T> va = a[t], vb = b[t];
                        const double pr0 = vsq * ((double)va.x * (double)vb.x + (double)va.y * (double)vb.y);
                        const double pi = vsq * ((double)va.y * (double)vb.x - (double)va.x * (double)vb.y);
                        const double w = any_sn0 ? ax.f(nx) * ax.f(ny) * ax.f(iz) : 0.0;
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            double pr = pr0;
                            if (cfg.sn0[c] != 0.0) pr -= cfg.sn0[c] * w;
                            if (cfg.source[c]) {
                                static_cast<cpx_t<T> *>(cfg.source[c])[t] =
                                    keep ? mk<T>((T)pr, (T)pi) : mk<T>((T)0, (T)0);
                                // the stored source is Hermitian on |k| < band: mult * Re sums the full space
                                if (keep) tot[c] += mult * (double)(T)pr;
                            }
                            if (bin >= 0) val[c] += mult * pr * y[c];
                        }
                    } else if (any_src) {
#pragma unroll
                        for (int c = 0; c < NC; ++c)
                            if (cfg.source[c]) static_cast<cpx_t<T> *>(cfg.source[c])[t] = mk<T>((T)0, (T)0);
                    }
                }
        }
        warp_run_add<NC>(bins, nbt, bin, val);
    }
    // source sums: per thread, then per warp, into bin nb of each configuration
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        if (!cfg.source[c]) continue;
        double x = tot[c];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0 && x != 0.0) atomicAdd(&bins[c * nbt + nb], x);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NC * nbt; i += blockDim.x) {
        const int c = i / nbt, j = i - c * nbt;
        if (bins[i] != 0.0 && (j < nb || cfg.source[c])) atomicAdd(&cfg.sums[c][2 * j], bins[i]);
    }
}

// --------------------------------------------------------- shell spectra
template <typename T>
__global__ void shell_spectra_kernel(const cpx_t<T> *A, const cpx_t<T> *B, int n, double L,
                                     EdgeSet edges, HarmTable harm, ItemTable items,
                                     cpx_t<T> *out, int64_t nh) {
    extern __shared__ double tbl[];
    AxisTable ax;
    fill_axis_table(ax, tbl, n, L, CNPC_COMP_NONE, 1);
    // edges, harmonics and items in shared memory: all are read at run-time indices
    const double *e = edges_to_shared(tbl + (n + 1), edges);
    cnpc_harmonic *sh = reinterpret_cast<cnpc_harmonic *>(tbl + (n + 1) + CNPC_MAX_EDGES);
    cnpc_shell_item *si = reinterpret_cast<cnpc_shell_item *>(sh + harm.n);
    for (int i = threadIdx.x; i < harm.n; i += blockDim.x) sh[i] = harm.h[i];
    for (int i = threadIdx.x; i < items.n; i += blockDim.x) si[i] = items.it[i];
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const cpx_t<T> zero = mk<T>((T)0, (T)0);
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += stride) {
        const Mode m = mode_of(t, n);
        const double kx = ax.kx(m.nx), ky = ax.kx(m.ny), kz = ax.kx(m.nz);
        const double kn = knorm_from(kx, ky, kz);
        const int bin = find_bin(kn, e, edges.n);
        if (bin < 0) {
            for (int j = 0; j < items.n; ++j) out[(int64_t)j * nh + t] = zero;
            continue;
        }
        const bool origin = kn == 0.0;
        const double ik = origin ? 0.0 : 1.0 / kn;
        const T x = (T)(kx * ik), y = (T)(ky * ik), z = (T)(kz * ik);
        for (int j = 0; j < items.n; ++j) {
            const cnpc_shell_item it = si[j];
            cpx_t<T> v = zero;
            if (it.bin == bin) {
                const cnpc_harmonic &h = sh[it.harmonic];
                cpx_t<T> Y = harmonic_eval<T>(h, x, y, z, origin);
                if (it.conj) Y.y = -Y.y;
                // phi = Re Y / Im Y (even l) or i Im Y / -i Re Y (odd l)
                cpx_t<T> phi;
                if ((h.l & 1) == 0)
                    phi = it.component == 0 ? mk<T>(Y.x, (T)0) : mk<T>(Y.y, (T)0);
                else
                    phi = it.component == 0 ? mk<T>((T)0, Y.y) : mk<T>((T)0, -Y.x);
                cpx_t<T> s;
                if (it.source == 0)
                    s = A[t];
                else if (it.source == 1)
                    s = B[t];
                else
                    s = mk<T>((T)1, (T)0);
                v = mk<T>(s.x * phi.x - s.y * phi.y, s.x * phi.y + s.y * phi.x);
            }
            out[(int64_t)j * nh + t] = v;
        }
    }
}

}  // namespace cnpc

using namespace cnpc;

extern "C" {

int cnpc_forward_finish_band(cnpc_ctx *ctx, int dtype, int n, double boxsize, void *d_spec,
                             const void *d_spec2, double scale, int comp, int window, double k0_value,
                             double band_kmax, void *d_band_out, double band_out_kmax, cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, d_spec != nullptr, "null spectrum");
    CNPC_REQUIRE(ctx, comp >= 0 && comp <= 3, "bad compensation kind");
    CNPC_REQUIRE(ctx, window >= 1 && window <= 4, "window must be 1..4");
    CNPC_REQUIRE(ctx, d_band_out != d_spec, "band output must not be the spectrum");
    const int64_t nq = (int64_t)(n / 2 + 1) * (n / 2 + 1) * (n / 2 + 1);  // sign orbits of the half spectrum
    const double inv_n3 = 1.0 / ((double)n * n * n);
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = 256;
    const int blocks = grid_for(ctx, nq, threads);
    const size_t tsm = 4 * sizeof(double) * (n + 1);  // k, compensation, interlacing phase
    if (dtype == CNPC_F32)
        forward_finish_kernel<float><<<blocks, threads, tsm, s>>>(
            (float2 *)d_spec, (const float2 *)d_spec2, n, boxsize, inv_n3, scale, comp, window,
            k0_value, band_kmax, (float2 *)d_band_out, band_out_kmax, nq);
    else
        forward_finish_kernel<double><<<blocks, threads, tsm, s>>>(
            (double2 *)d_spec, (const double2 *)d_spec2, n, boxsize, inv_n3, scale, comp, window,
            k0_value, band_kmax, (double2 *)d_band_out, band_out_kmax, nq);
    return check_launch(ctx, "forward_finish_kernel");
}

int cnpc_forward_finish(cnpc_ctx *ctx, int dtype, int n, double boxsize, void *d_spec,
                        const void *d_spec2, double scale, int comp, int window, double k0_value,
                        double band_kmax, cnpc_stream_t stream) {
    return cnpc_forward_finish_band(ctx, dtype, n, boxsize, d_spec, d_spec2, scale, comp, window, k0_value,
                                    band_kmax, nullptr, 0.0, stream);
}

int cnpc_kbin_counts(cnpc_ctx *ctx, int n, double boxsize, const double *h_edges, int nedges,
                     double *d_counts, double *d_ksum, cnpc_stream_t stream) {
    int st = check_common(ctx, CNPC_F64, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, d_counts && d_ksum, "null output");
    EdgeSet es;
    st = load_edges(ctx, h_edges, nedges, &es);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = nedges - 1;
    st = check_cuda(ctx, cudaMemsetAsync(d_counts, 0, sizeof(double) * nb, s), "memset");
    if (st) return st;
    st = check_cuda(ctx, cudaMemsetAsync(d_ksum, 0, sizeof(double) * nb, s), "memset");
    if (st) return st;
    const QuadIter qi = quad_iter(n, boxsize, h_edges[nedges - 1]);
    const int threads = 256;
    kbin_counts_kernel<<<grid_for(ctx, qi.count, threads), threads, (n + 1 + 2 * nb + nedges) * sizeof(double), s>>>(
        n, boxsize, es, d_counts, d_ksum, qi);
    return check_launch(ctx, "kbin_counts_kernel");
}

int cnpc_pk_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                 const void *d_spec_b, const double *h_edges, int nedges, const int *h_poles,
                 int npoles, const double *h_los, double *d_sums, cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, d_spec_a && d_spec_b && d_sums && h_poles && h_los, "null argument");
    CNPC_REQUIRE(ctx, npoles >= 1 && npoles <= CNPC_MAX_POLES, "npoles out of range (1..8)");
    EdgeSet es;
    st = load_edges(ctx, h_edges, nedges, &es);
    if (st) return st;
    PoleSet ps;
    ps.n = npoles;
    for (int i = 0; i < npoles; ++i) {
        CNPC_REQUIRE(ctx, h_poles[i] >= 0 && h_poles[i] <= 16, "pole out of range (0..16)");
        ps.l[i] = h_poles[i];
    }
    for (int d = 0; d < 3; ++d) ps.los[d] = h_los[d];
    const int nb = nedges - 1;
    cudaStream_t s = (cudaStream_t)stream;
    st = check_cuda(ctx, cudaMemsetAsync(d_sums, 0, sizeof(double) * nb * npoles, s), "memset");
    if (st) return st;
    const BandIter bi = band_iter(n, boxsize, h_edges[nedges - 1]);
    const int64_t rq = bi.R < 0 ? n / 2 : bi.R;
    const int64_t nh = (rq + 1) * (rq + 1) * (rq + 1);  // sign-folded items
    const int threads = 256;
    const size_t smem = sizeof(double) * (n + 1 + nb * npoles + nedges);
    if (dtype == CNPC_F32)
        pk_bins_kernel<float><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            (const float2 *)d_spec_a, (const float2 *)d_spec_b, n, boxsize, es, ps, d_sums, bi);
    else
        pk_bins_kernel<double><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            (const double2 *)d_spec_a, (const double2 *)d_spec_b, n, boxsize, es, ps, d_sums, bi);
    return check_launch(ctx, "pk_bins_kernel");
}

static int run_sn_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                       const void *d_spec_b, double volume_sq, int window, int ncfg, const double *h_sn0,
                       const cnpc_harmonic *const *h_yl0, const double *h_edges, int nedges,
                       double *const *d_sums, void *const *d_source, double band_kmax, cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, d_spec_a && d_spec_b && h_sn0 && h_yl0 && d_sums && d_source, "null argument");
    CNPC_REQUIRE(ctx, window >= 1 && window <= 4, "window must be 1..4");
    CNPC_REQUIRE(ctx, ncfg >= 1 && ncfg <= kSnMaxCfg, "ncfg must be 1..2");
    EdgeSet es;
    st = load_edges(ctx, h_edges, nedges, &es);
    if (st) return st;
    SnCfg cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    const int nb = nedges - 1;
    cudaStream_t s = (cudaStream_t)stream;
    for (int c = 0; c < ncfg; ++c) {
        CNPC_REQUIRE(ctx, d_sums[c] != nullptr, "null sums");
        cfg.sn0[c] = h_sn0[c];
        if (h_yl0[c]) {
            cfg.yl0[c] = *h_yl0[c];
            cfg.use_y[c] = 1;
            CNPC_REQUIRE(ctx, cfg.yl0[c].l >= 0 && cfg.yl0[c].l <= 8 && cfg.yl0[c].m == 0, "Y_L0 harmonic expected");
        }
        cfg.sums[c] = d_sums[c];
        cfg.source[c] = d_source[c];
        const int nbt = d_source[c] ? nb + 1 : nb;
        st = check_cuda(ctx, cudaMemsetAsync(d_sums[c], 0, sizeof(double) * 2 * nbt, s), "memset");
        if (st) return st;
    }
    const int64_t nq = (int64_t)(n / 2 + 1) * (n / 2 + 1) * (n / 2 + 1);  // sign-folded items
    const int threads = 256;
    const size_t smem = sizeof(double) * (2 * (n + 1) + ncfg * (nb + 1) + nedges);
    const int grid = grid_for(ctx, nq, threads);
#define CNPC_SN_LAUNCH(T_, NC_)                                                                          \
    sn_bins_kernel<T_, NC_><<<grid, threads, smem, s>>>((const cpx_t<T_> *)d_spec_a,                     \
                                                       (const cpx_t<T_> *)d_spec_b, n, boxsize, volume_sq, \
                                                       window, es, cfg, band_kmax, nq)
    if (dtype == CNPC_F32) {
        if (ncfg == 1) CNPC_SN_LAUNCH(float, 1);
        else CNPC_SN_LAUNCH(float, 2);
    } else {
        if (ncfg == 1) CNPC_SN_LAUNCH(double, 1);
        else CNPC_SN_LAUNCH(double, 2);
    }
#undef CNPC_SN_LAUNCH
    return check_launch(ctx, "sn_bins_kernel");
}

int cnpc_sn_bins(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                 const void *d_spec_b, double volume_sq, double sn0, int window,
                 const cnpc_harmonic *h_yl0, const double *h_edges, int nedges, double *d_sums,
                 void *d_source, double band_kmax, cnpc_stream_t stream) {
    return run_sn_bins(ctx, dtype, n, boxsize, d_spec_a, d_spec_b, volume_sq, window, 1, &sn0, &h_yl0, h_edges,
                       nedges, &d_sums, &d_source, band_kmax, stream);
}

int cnpc_sn_bins_multi(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                       const void *d_spec_b, double volume_sq, int window, int ncfg, const double *h_sn0,
                       const cnpc_harmonic *const *h_yl0, const double *h_edges, int nedges,
                       double *const *d_sums, void *const *d_source, double band_kmax, cnpc_stream_t stream) {
    return run_sn_bins(ctx, dtype, n, boxsize, d_spec_a, d_spec_b, volume_sq, window, ncfg, h_sn0, h_yl0, h_edges,
                       nedges, d_sums, d_source, band_kmax, stream);
}

int cnpc_shell_spectra(cnpc_ctx *ctx, int dtype, int n, double boxsize, const void *d_spec_a,
                       const void *d_spec_b, const double *h_edges, int nedges,
                       const cnpc_harmonic *h_harmonics, int nharmonics,
                       const cnpc_shell_item *h_items, int nitems, void *d_out,
                       cnpc_stream_t stream) {
    int st = check_common(ctx, dtype, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, d_out != nullptr, "null output");
    CNPC_REQUIRE(ctx, nitems >= 1 && nitems <= CNPC_MAX_ITEMS, "nitems out of range (1..256)");
    CNPC_REQUIRE(ctx, nharmonics >= 1 && nharmonics <= CNPC_MAX_HARMONICS, "nharmonics out of range");
    CNPC_REQUIRE(ctx, h_harmonics && h_items, "null table");
    EdgeSet es;
    st = load_edges(ctx, h_edges, nedges, &es);
    if (st) return st;
    HarmTable ht;
    ht.n = nharmonics;
    for (int i = 0; i < nharmonics; ++i) {
        const cnpc_harmonic &h = h_harmonics[i];
        CNPC_REQUIRE(ctx, h.l >= 0 && h.l <= 8 && h.m >= -h.l && h.m <= h.l, "bad harmonic (l<=8, |m|<=l)");
        ht.h[i] = h;
    }
    ItemTable itab;
    itab.n = nitems;
    for (int j = 0; j < nitems; ++j) {
        const cnpc_shell_item &it = h_items[j];
        CNPC_REQUIRE(ctx, it.bin >= 0 && it.bin < nedges - 1, "item bin out of range");
        CNPC_REQUIRE(ctx, it.harmonic >= 0 && it.harmonic < nharmonics, "item harmonic out of range");
        CNPC_REQUIRE(ctx, it.component == 0 || it.component == 1, "item component must be 0/1");
        CNPC_REQUIRE(ctx, it.source >= 0 && it.source <= 2, "item source must be 0..2");
        CNPC_REQUIRE(ctx, it.source != 0 || d_spec_a, "item needs spectrum A");
        CNPC_REQUIRE(ctx, it.source != 1 || d_spec_b, "item needs spectrum B");
        itab.it[j] = it;
    }
    const int64_t nh = half_modes(n);
    const int threads = 256;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = (n + 1 + CNPC_MAX_EDGES) * sizeof(double) + nharmonics * sizeof(cnpc_harmonic) +
                        nitems * sizeof(cnpc_shell_item);  // < 48 KB for n <= 2048
    if (dtype == CNPC_F32)
        shell_spectra_kernel<float><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            (const float2 *)d_spec_a, (const float2 *)d_spec_b, n, boxsize, es, ht, itab,
            (float2 *)d_out, nh);
    else
        shell_spectra_kernel<double><<<grid_for(ctx, nh, threads), threads, smem, s>>>(
            (const double2 *)d_spec_a, (const double2 *)d_spec_b, n, boxsize, es, ht, itab,
            (double2 *)d_out, nh);
    return check_launch(ctx, "shell_spectra_kernel");
}

}  // extern "C"
