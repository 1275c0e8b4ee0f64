// Shared device helpers for the CosmoNPC B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cosmonpc_b200.h"

namespace cnpc {

// np.pi as a double (the reference's k vectors are built from it).
constexpr double kPi = 3.141592653589793;

template <typename T> struct cpx_of;
template <> struct cpx_of<float> { using type = float2; };
template <> struct cpx_of<double> { using type = double2; };
template <typename T> using cpx_t = typename cpx_of<T>::type;

template <typename T> __host__ __device__ inline cpx_t<T> mk(T r, T i) {
    cpx_t<T> c;
    c.x = r;
    c.y = i;
    return c;
}

// Geometry of one half-spectrum mode (cuFFT R2C layout n x n x (n/2+1)).
struct Mode {
    int nx, ny, nz;  // integer wave numbers, FFT order (Nyquist negative in x, y)
    int mult;        // full-space modes represented: 1 on the iz = 0 and iz = n/2 planes
};

// q = u / d and *rem = u % d for 0 <= u < 2^31, d >= 1, without an integer
// division: trunc(u * RN(1/d)) in FP64 is within one of the quotient (the
// reciprocal and the product are accurate to 2^-53 relative), and one
// correction step makes it exact.  The reciprocal of a loop-invariant d is
// hoisted out of the caller's loop.
__device__ __forceinline__ uint32_t udiv31(uint32_t u, uint32_t d, uint32_t *rem) {
    uint32_t q = (uint32_t)((double)u * (1.0 / (double)d));
    int64_t r = (int64_t)u - (int64_t)q * d;
    if (r < 0) {
        --q;
        r += d;
    } else if (r >= d) {
        ++q;
        r -= d;
    }
    *rem = (uint32_t)r;
    return q;
}

__device__ inline Mode mode_of(int64_t t, int n) {
    const int nz2 = n / 2 + 1;
    Mode m;
    int iz, iy, ix;
    if (t < ((int64_t)1 << 31)) {  // every mode of meshes up to 1024^3
        uint32_t rz, ry;
        const uint32_t r = udiv31((uint32_t)t, (uint32_t)nz2, &rz);
        ix = (int)udiv31(r, (uint32_t)n, &ry);
        iz = (int)rz;
        iy = (int)ry;
    } else {
        iz = (int)(t % nz2);
        const int64_t r = t / nz2;
        iy = (int)(r % n);
        ix = (int)(r / n);
    }
    m.nx = ix >= n / 2 ? ix - n : ix;
    m.ny = iy >= n / 2 ? iy - n : iy;
    m.nz = iz;
    m.mult = (iz == 0 || 2 * iz == n) ? 1 : 2;
    return m;
}

// k = (2 n) * pi / L, in the operation order of the restated pmesh k vectors.
__device__ inline double kcomp(int n_int, double boxsize) {
    return __ddiv_rn(__dmul_rn((double)(2 * n_int), kPi), boxsize);
}

// |k| = sqrt((kx^2 + ky^2) + kz^2) with every operation rounded separately
// (no FMA contraction), which reproduces numpy's value bit for bit.
__device__ inline double knorm_from(double kx, double ky, double kz) {
    double s = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    return __dsqrt_rn(s);
}

__device__ inline double knorm_exact(const Mode &m, double boxsize, double *kx, double *ky,
                                     double *kz) {
    *kx = kcomp(m.nx, boxsize);
    *ky = kcomp(m.ny, boxsize);
    *kz = kcomp(m.nz, boxsize);
    double s = __dadd_rn(__dadd_rn(__dmul_rn(*kx, *kx), __dmul_rn(*ky, *ky)), __dmul_rn(*kz, *kz));
    return __dsqrt_rn(s);
}

// Bin b with e[b] <= v < e[b+1], or -1 (searchsorted(..., "right") - 1 on the
// valid range [e[0], e[last])).  The guess from an even spacing is corrected
// against the actual edges, so any increasing edges give the exact answer.
__device__ inline int find_bin(double v, const double *e, int nedges) {
    if (!(v >= e[0]) || !(v < e[nedges - 1])) return -1;
    const int nb = nedges - 1;
    // first guess from the mean bin width (a loop-invariant reciprocal, hoisted
    // by the compiler); the two walks below make the bin exact
    int b = (int)((v - e[0]) * ((double)nb / (e[nb] - e[0])));
    b = b < 0 ? 0 : (b >= nb ? nb - 1 : b);
    while (b > 0 && v < e[b]) --b;
    while (b < nb - 1 && v >= e[b + 1]) ++b;
    return b;
}

// Per-axis values shared by every mode of a block: the exact wave numbers
// k(j) for integer j in [-n/2, n/2] and, optionally, the per-axis factor of a
// separable window compensation.  Filled cooperatively at kernel start.
struct AxisTable {
    double *k;   // k[j + n/2]
    double *cf;  // cf[j + n/2] or nullptr
    int half;
    __device__ double kx(int j) const { return k[j + half]; }
    __device__ double f(int j) const { return cf[j + half]; }
};

// sinc(w / 2) = sin(w/2) / (w/2), 1 at w = 0 (np.sinc(0.5 w / pi)).
__device__ inline double sinc_half(double w) {
    if (w == 0.0) return 1.0;
    double h = 0.5 * w;
    return sin(h) / h;
}

__device__ inline double ipow(double x, int p) {
    double r = 1.0;
    for (int i = 0; i < p; ++i) r *= x;
    return r;
}

// C_p(s) of the shot-noise window, s = sin^2(w/2)  (math_evaluator.py:251-309).
__device__ inline double cwin(int p, double s) {
    if (p == 2) return 1.0 - 2.0 / 3 * s;
    if (p == 3) return 1.0 - s + 2.0 / 15 * s * s;
    if (p == 4) return 1.0 - 4.0 / 3.0 * s + 2.0 / 5.0 * s * s - 4.0 / 315.0 * s * s * s;
    return 1.0;
}

// One axis's factor of the separable compensation (comp_factor = product of
// the three axes' factors).
__device__ inline double comp_axis(int kind, int p, double w) {
    if (kind == CNPC_COMP_SINC) return 1.0 / ipow(sinc_half(w), p);
    if (p == 1) return 1.0;
    if (kind == CNPC_COMP_SHOTNOISE) {
        const double s = sin(0.5 * w);
        return 1.0 / sqrt(cwin(p, s * s));
    }
    if (kind == CNPC_COMP_BKNOISE) {
        const double s = sin(0.5 * w);
        const double t = ipow(sinc_half(w), p);
        return cwin(p, s * s) / (t * t);
    }
    return 1.0;
}

// Fill an AxisTable in shared memory (all threads of the block call this,
// then __syncthreads()).
__device__ inline void fill_axis_table(AxisTable &t, double *smem, int n, double boxsize, int kind, int p) {
    t.half = n / 2;
    t.k = smem;
    t.cf = kind == CNPC_COMP_NONE ? nullptr : smem + (n + 1);
    const double H = boxsize / n;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        const double k = kcomp(i - n / 2, boxsize);
        t.k[i] = k;
        if (t.cf) t.cf[i] = comp_axis(kind, p, k * H);
    }
}

// Multiplicative compensation factor at circular coordinates w = k H.
__device__ inline double comp_factor(int kind, int p, double wx, double wy, double wz) {
    if (kind == CNPC_COMP_NONE) return 1.0;
    double w[3] = {wx, wy, wz};
    double f = 1.0;
    for (int d = 0; d < 3; ++d) {
        if (kind == CNPC_COMP_SINC) {
            f /= ipow(sinc_half(w[d]), p);
        } else if (kind == CNPC_COMP_SHOTNOISE) {
            if (p == 1) continue;
            double s = sin(0.5 * w[d]);
            f /= sqrt(cwin(p, s * s));
        } else if (kind == CNPC_COMP_BKNOISE) {
            if (p == 1) continue;
            double s = sin(0.5 * w[d]);
            double t = ipow(sinc_half(w[d]), p);
            f *= cwin(p, s * s) / (t * t);
        }
    }
    return f;
}

// Spherical harmonic (see cnpc_harmonic) at unit vector (x, y, z); `origin`
// selects the k = 0 value.
template <typename T>
__device__ inline cpx_t<T> harmonic_eval(const cnpc_harmonic &h, T x, T y, T z, bool origin) {
    if (origin) return mk<T>((T)h.origin_re, (T)h.origin_im);
    const int ma = h.m < 0 ? -h.m : h.m;
    const int deg = h.l - ma;
    T p = (T)h.coef[deg];
    for (int i = deg - 1; i >= 0; --i) p = p * z + (T)h.coef[i];
    p *= (T)h.norm;
    T re = (T)1, im = (T)0;
    for (int i = 0; i < ma; ++i) {
        T nr = re * x - im * y;
        T ni = re * y + im * x;
        re = nr;
        im = ni;
    }
    re *= p;
    im *= p;
    if (h.m < 0) {
        T s = (ma & 1) ? (T)-1 : (T)1;
        re = s * re;
        im = -s * im;
    }
    return mk<T>(re, im);
}

}  // namespace cnpc
