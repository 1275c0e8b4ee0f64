// Band-limited shell fields: synthesis of mask_bin(|k|) * phi(k) * src(k)
// fused with its inverse 3-D FFT, FP32.
//
// A shell spectrum of the bispectrum is non-zero only for |k| < k_top, and the
// reference's own rule 2 k_max < k_Nyquist puts every such mode inside
// |n_x|, |n_y|, |n_z| < n/4.  The inverse transform therefore runs on the
// band only:
//   pass 1 (x): for each in-band column (n_y, n_z) the n-point inverse DFT
//     along x of the synthesised column, written compactly as
//     A[x][n_y + n/4][n_z] (n x n/2 x n/4 complex per field);
//   pass 2 (y then z, per x-slab in shared memory): inverse DFT along y of the
//     n/4 columns, then the real output along z from the n_z < n/4 half-line
//     (Hermitian extension), two rows per complex transform; each x-slab of
//     the real field is written once.
// An n-point inverse DFT whose input is confined to |k| < n/4 is computed as
// two n/2-point FFTs (even and odd outputs; the odd one with input twiddles
// e^{2 pi i s / n}) and the output phase (-1)^m (-i)^r of the shift by n/4.
// The n/2-point FFT is done by a team of T threads holding V values each: a
// V-point DFT in registers, twiddles, one shared-memory exchange and T-point
// DFTs.  n = 64, 128, 256 use V = 16 and T = n/32; n = 192 (M = 96, which has
// the factor 3) uses V = 24 (8 x 3 in registers) and T = 4.  Twiddles come
// from an FP64-computed table rounded to FP32.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "bins.cuh"

namespace cnpc {

namespace {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }      // i a
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }     // -i a

// inverse DFTs (kernel e^{+2 pi i jk / N}) in registers, in place
__device__ __forceinline__ void idft2(float2 &a, float2 &b) {
    const float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

__device__ __forceinline__ void idft4(float2 &a, float2 &b, float2 &c, float2 &d) {
    const float2 s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = mul_i(csub(b, d));
    a = cadd(s0, s2);
    c = csub(s0, s2);
    b = cadd(s1, s3);
    d = csub(s1, s3);
}

constexpr float kC8 = 0.70710678118654752440f;   // cos(pi/4)
constexpr float kC16 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kS16 = 0.38268343236508977173f;  // sin(pi/8)

__device__ __forceinline__ void idft8(float2 *v) {
    // j = 2 j1 + j2: two 4-point DFTs, twiddle W8^{k1} on the odd half, 2-point DFTs
    idft4(v[0], v[2], v[4], v[6]);
    idft4(v[1], v[3], v[5], v[7]);
    // v[1], v[3], v[5], v[7] hold k1 = 0..3 of the odd half
    v[3] = cmul(v[3], make_float2(kC8, kC8));
    v[5] = mul_i(v[5]);
    v[7] = cmul(v[7], make_float2(-kC8, kC8));
    float2 o[8];
    for (int k1 = 0; k1 < 4; ++k1) {
        float2 a = v[2 * k1], b = v[2 * k1 + 1];
        idft2(a, b);
        o[k1] = a;
        o[k1 + 4] = b;
    }
    for (int i = 0; i < 8; ++i) v[i] = o[i];
}

// W16^m, m = 0..15
__device__ __forceinline__ float2 w16(int m) {
    switch (m & 15) {
        case 0: return make_float2(1.f, 0.f);
        case 1: return make_float2(kC16, kS16);
        case 2: return make_float2(kC8, kC8);
        case 3: return make_float2(kS16, kC16);
        case 4: return make_float2(0.f, 1.f);
        case 5: return make_float2(-kS16, kC16);
        case 6: return make_float2(-kC8, kC8);
        case 7: return make_float2(-kC16, kS16);
        case 8: return make_float2(-1.f, 0.f);
        case 9: return make_float2(-kC16, -kS16);
        case 10: return make_float2(-kC8, -kC8);
        case 11: return make_float2(-kS16, -kC16);
        case 12: return make_float2(0.f, -1.f);
        case 13: return make_float2(kS16, -kC16);
        case 14: return make_float2(kC8, -kC8);
        default: return make_float2(kC16, -kS16);
    }
}

__device__ __forceinline__ void idft16(float2 *v) {
    // j = 4 j1 + j2; step 1: 4-point DFTs over j1 for each j2
#pragma unroll
    for (int j2 = 0; j2 < 4; ++j2) idft4(v[j2], v[4 + j2], v[8 + j2], v[12 + j2]);
    // now v[4 k1 + j2] = Y[j2][k1]; twiddle W16^{j2 k1}
#pragma unroll
    for (int j2 = 1; j2 < 4; ++j2)
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) v[4 * k1 + j2] = cmul(v[4 * k1 + j2], w16(j2 * k1));
    // step 3: 4-point DFT over j2 for each k1 -> X[k1 + 4 k2]
    float2 o[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        float2 a = v[4 * k1], b = v[4 * k1 + 1], c = v[4 * k1 + 2], d = v[4 * k1 + 3];
        idft4(a, b, c, d);
        o[k1] = a;
        o[k1 + 4] = b;
        o[k1 + 8] = c;
        o[k1 + 12] = d;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = o[i];
}

// 3-point inverse DFT: with W = e^{2 pi i / 3} = -1/2 + i sqrt(3)/2,
// X1 = a - (b + c)/2 + i sqrt(3)/2 (b - c) and X2 its partner with -i.
constexpr float kS3 = 0.86602540378443864676f;  // sin(pi/3)
__device__ __forceinline__ void idft3(float2 &a, float2 &b, float2 &c) {
    const float2 s = cadd(b, c), d = csub(b, c);
    const float2 h = make_float2(a.x - 0.5f * s.x, a.y - 0.5f * s.y);
    const float2 r = make_float2(-kS3 * d.y, kS3 * d.x);  // i sqrt(3)/2 (b - c)
    a = cadd(a, s);
    b = cadd(h, r);
    c = csub(h, r);
}

constexpr float kC24 = 0.96592582628906828675f;  // cos(pi/12)
constexpr float kS24 = 0.25881904510252076235f;  // sin(pi/12)

// W24^m = e^{2 pi i m / 24}, m = 0..14 (the products j2 k1 of idft24)
__device__ __forceinline__ float2 w24(int m) {
    switch (m) {
        case 0: return make_float2(1.f, 0.f);
        case 1: return make_float2(kC24, kS24);
        case 2: return make_float2(kS3, 0.5f);
        case 3: return make_float2(kC8, kC8);
        case 4: return make_float2(0.5f, kS3);
        case 5: return make_float2(kS24, kC24);
        case 6: return make_float2(0.f, 1.f);
        case 7: return make_float2(-kS24, kC24);
        case 8: return make_float2(-0.5f, kS3);
        case 10: return make_float2(-kS3, 0.5f);
        case 12: return make_float2(-1.f, 0.f);
        default: return make_float2(-kS3, -0.5f);  // 14
    }
}

__device__ __forceinline__ void idft24(float2 *v) {
    // j = 3 j1 + j2, k = k1 + 8 k2: W24^{jk} = W8^{j1 k1} W24^{j2 k1} W3^{j2 k2}
    float2 a[3][8];
#pragma unroll
    for (int j2 = 0; j2 < 3; ++j2) {
#pragma unroll
        for (int j1 = 0; j1 < 8; ++j1) a[j2][j1] = v[3 * j1 + j2];
        idft8(a[j2]);
    }
#pragma unroll
    for (int j2 = 1; j2 < 3; ++j2)
#pragma unroll
        for (int k1 = 1; k1 < 8; ++k1) a[j2][k1] = cmul(a[j2][k1], w24(j2 * k1));
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) {
        idft3(a[0][k1], a[1][k1], a[2][k1]);
        v[k1] = a[0][k1];
        v[k1 + 8] = a[1][k1];
        v[k1 + 16] = a[2][k1];
    }
}

// V-point inverse DFT in registers (natural order out)
template <int V> __device__ __forceinline__ void idft_regs(float2 *v) {
    if constexpr (V == 16)
        idft16(v);
    else
        idft24(v);
}

// Exchange slots of one team: V rows of T float2, element (k1, c) at
// k1 T + (c ^ ((k1 / (V / T)) % T)), and a team stride of T (mod 16) float2.
// The row writes (fixed k1, c = t) and the transposed reads (k1 = t V/T + q,
// fixed c) of the teams of a warp then hit every bank pair exactly twice for
// V = 16: no bank conflicts for T = 2, 4, 8.
template <int T, int V = 16> struct Exch {
    static constexpr int kStride = (V + 1) * T;
};

// Per-thread twiddles of team_fft, [k1 - 1][t] = W_M^{t k1} (k1 = 1..V-1): the
// T threads of a team read T consecutive slots.
template <int T, int V = 16> __host__ __device__ constexpr int team_twiddles() { return (V - 1) * T; }
template <int T, int V = 16> __device__ __forceinline__ void fill_team_twiddles(float2 *twt, const float2 *tw) {
    for (int e = threadIdx.x; e < (V - 1) * T; e += blockDim.x) {
        const int k1 = e / T + 1, t = e % T;
        twt[e] = tw[2 * ((t * k1) % (V * T))];
    }
}

// Team FFT of size M = V T (inverse).  On entry thread t of the team holds
// u[j] = x[T j + t]; on exit it holds X[k1 + V k2] for k1 = t (V/T) + q
// (q < V/T), k2 < T, stored as u[q * T + k2].  ex: the team's exchange slots
// (Exch<T, V>); twt: the per-thread twiddle table (fill_team_twiddles).
template <int T, int V = 16>
__device__ __forceinline__ void team_fft(float2 *u, int t, float2 *ex, const float2 *twt, unsigned mask) {
    static_assert(V % T == 0, "V must be a multiple of T");
    constexpr int Q = V / T;
    idft_regs<V>(u);
#pragma unroll
    for (int k1 = 1; k1 < V; ++k1) u[k1] = cmul(u[k1], twt[(k1 - 1) * T + t]);
#pragma unroll
    for (int k1 = 0; k1 < V; ++k1) ex[k1 * T + (t ^ ((k1 / Q) % T))] = u[k1];
    __syncwarp(mask);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int k1 = t * Q + q;
        float2 w[T];
#pragma unroll
        for (int i = 0; i < T; ++i) w[i] = ex[k1 * T + (i ^ t)];
        if (T == 2) idft2(w[0], w[1]);
        if (T == 4) idft4(w[0], w[1], w[2], w[3]);
        if (T == 8) idft8(w);
#pragma unroll
        for (int i = 0; i < T; ++i) u[q * T + i] = w[i];
    }
    __syncwarp(mask);
}

// output index m (of the M-point transform) held in u[q T + k2]
template <int T, int V = 16>
__device__ __forceinline__ int team_out_index(int t, int q, int k2) {
    return (t * (V / T) + q) + V * k2;
}

// (-1)^m (-i)^r phase of the shift by n/4 for output position x = 2 m + r
__device__ __forceinline__ float2 shift_phase(float2 v, int m, int r) {
    if (r) v = mul_mi(v);
    if (m & 1) v = make_float2(-v.x, -v.y);
    return v;
}

struct ShellItemsDev {
    int n;
    cnpc_shell_item it[CNPC_MAX_ITEMS];
    // band of the item (with a relative slack of 1e-9 so that FP64 rounding of
    // |k| never puts a mode outside it): no mode has |n_d| > rmax or
    // n_y^2 + n_z^2 > r2max
    int rmax[CNPC_MAX_ITEMS];
    int r2max[CNPC_MAX_ITEMS];
};

// Pass 1 writes the (s, chunk) tile of an item only when it can hold a mode of
// the shell; pass 2 reads exactly those tiles (others are zero).
__device__ __forceinline__ bool tile_live(int ny, int kz0, int r2max) { return ny * ny + kz0 * kz0 <= r2max; }

}  // namespace

// ------------------------------------------------------------ passes
// Work layout per item: A[x][s][n_z] (pass 1 output, s = n_y + n/4) and
// B[x][y][n_z] (pass 2 output); n_z < n/4 throughout.
constexpr int kColThreads = 128;   // 16 teams of 8 (n = 256)
// unit-spectrum shells: planes x > N/2 written as reflections by the y/z
// passes (yz_mirror), so pass 1 does not store them
constexpr bool kMirrorUnitShells = true;
constexpr int kKC = 16;            // n_z columns per block in passes 1 and 2

__device__ __forceinline__ void fill_twiddles(float2 *tw, int N) {
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * j / N, &sn, &cs);
        tw[j] = make_float2((float)cs, (float)sn);
    }
}

__device__ __forceinline__ unsigned team_mask(int T) {
    return (((1u << T) - 1u) << ((threadIdx.x & 31) & ~(T - 1)));
}

// Pass 1: block (s, chunk, item) synthesises kKC in-band columns over n_x
// from the source spectrum, transforms them along x and writes
// A[x][s][chunk].
template <int T, int V>
__global__ void __launch_bounds__(kColThreads) shell_column_kernel(
    const float2 *__restrict__ Aspec, const float2 *__restrict__ Bspec, int n, double L, EdgeSet edges,
    HarmTable harm, ShellItemsDev items, float2 *__restrict__ dst) {
    constexpr int M = V * T, N = 2 * M, H = M / 2;
    constexpr int KC = (kKC < H) ? kKC : H;
    constexpr int LDC = KC + 1;
    constexpr int NCH = H / KC;
    extern __shared__ float4 smem4[];
    float2 *in = reinterpret_cast<float2 *>(smem4);  // [M][LDC]
    float2 *out = in + M * LDC;                      // [N][LDC]
    float2 *tw = out + N * LDC;                      // [N]
    float2 *ex = tw + N;                             // [teams][Exch<T, V>::kStride]
    float2 *twt = ex + (kColThreads / T) * Exch<T, V>::kStride;               // [(V - 1) T]
    double *kt = reinterpret_cast<double *>(twt + team_twiddles<T, V>());     // [n + 1]
    double *se = kt + (n + 1);                                                 // [edges.n]
    const int nitems = items.n;
    const int item = blockIdx.x % nitems;
    const int chunk = (blockIdx.x / nitems) % NCH;
    const int row = blockIdx.x / (nitems * NCH);  // s - 1
    const int kz0 = chunk * KC;
    if (!tile_live(row + 1 - H, kz0, items.r2max[item])) return;
    fill_twiddles(tw, N);
    {
        for (int i = threadIdx.x; i <= n; i += blockDim.x) kt[i] = kcomp(i - n / 2, L);
        // edges and the harmonic are read at run-time indices: shared copies
        edges_to_shared(se, edges);
        __shared__ cnpc_harmonic hm;
        const cnpc_shell_item it = items.it[item];
        if (threadIdx.x == 0) hm = harm.h[it.harmonic];
        __syncthreads();
        fill_team_twiddles<T, V>(twt, tw);  // first read after the barrier below
        const int s = row + 1;
        const int ny = s - H;
        const int iy = ny < 0 ? ny + n : ny;
        const int nh2 = n / 2 + 1;
        for (int e = threadIdx.x; e < M * KC; e += blockDim.x) {
            const int xs = e / KC, nz = kz0 + e % KC;
            float2 v = make_float2(0.f, 0.f);
            if (xs > 0) {
                const int nx = xs - H;
                const int ix = nx < 0 ? nx + n : nx;
                const double kx = kt[nx + n / 2], ky = kt[ny + n / 2], kz = kt[nz + n / 2];
                const double kn = knorm_from(kx, ky, kz);
                if (find_bin(kn, se, edges.n) == it.bin) {
                    const bool origin = kn == 0.0;
                    const double ik = origin ? 0.0 : 1.0 / kn;
                    float2 Y = harmonic_eval<float>(hm, (float)(kx * ik), (float)(ky * ik), (float)(kz * ik), origin);
                    if (it.conj) Y.y = -Y.y;
                    float2 phi;
                    if ((hm.l & 1) == 0)
                        phi = it.component == 0 ? make_float2(Y.x, 0.f) : make_float2(Y.y, 0.f);
                    else
                        phi = it.component == 0 ? make_float2(0.f, Y.y) : make_float2(0.f, -Y.x);
                    const int64_t t = ((int64_t)ix * n + iy) * nh2 + nz;
                    float2 sv;
                    if (it.source == 0)
                        sv = Aspec[t];
                    else if (it.source == 1)
                        sv = Bspec[t];
                    else
                        sv = make_float2(1.f, 0.f);
                    v = cmul(sv, phi);
                }
            }
            in[xs * LDC + (nz - kz0)] = v;
        }
    }
    __syncthreads();
    const int team = threadIdx.x / T, t = threadIdx.x % T, nteams = kColThreads / T;
    const unsigned mask = team_mask(T);
    float2 *tex = ex + team * Exch<T, V>::kStride;
    for (int job = team; job < 2 * KC; job += nteams) {
        const int c = job >> 1, r = job & 1;
        float2 u[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const int slot = T * j + t;
            float2 v = in[slot * LDC + c];
            if (r) v = cmul(v, tw[slot]);
            u[j] = v;
        }
        team_fft<T, V>(u, t, tex, twt, mask);
#pragma unroll
        for (int q = 0; q < V / T; ++q)
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) {
                const int m = team_out_index<T, V>(t, q, k2);
                out[(2 * m + r) * LDC + c] = shift_phase(u[q * T + k2], m, r);
            }
    }
    __syncthreads();
    // A[x][s][kz]; a unit-spectrum item's planes x > N/2 are never read
    float2 *d = dst + (size_t)item * N * M * H + (size_t)(row + 1) * H + kz0;
    const size_t stride = (size_t)M * H;
    const int np = (kMirrorUnitShells && items.it[item].source == 2) ? N / 2 + 1 : N;
    for (int e = threadIdx.x; e < np * KC; e += blockDim.x) {
        const int p = e / KC, c = e % KC;
        d[p * stride + c] = out[p * LDC + c];
    }
}

// Passes 2+3 fused: block (x, y parity ry, item).  The y transform of the n/4
// columns of A[x] (read from global memory) yields the rows y = 2m + ry,
// m < n/2, of B[x] into shared memory; the z pass then turns row pairs
// (m1, m2) into two real rows of the field through one complex transform of
// v(k_z) = B1~(k_z) + i B2~(k_z), B~(-k_z) = conj B(k_z), B~(0) = Re B(0).
// Thread t of a team ends the z pass holding z = 2Q t + c + 2V k2 (c < 2Q,
// Q = V/T) of both rows, written as float4 runs without staging.
// V = 16: 256 threads, 2 blocks per SM.  V = 24 (n = 192) keeps 24 values
// per FFT and 48 results of the z pass per thread: 48 teams of 4 (one round
// for the n/4 = 48 columns of the y pass and the 48 row pairs of the z pass),
// 2 blocks per SM, so the register limit is 170.
template <int T, int V = 16> struct YZLayout {
    static constexpr int THREADS = V == 16 ? 256 : 192;
    static constexpr int MIN_BLOCKS = 2;
    static constexpr int M = V * T, N = 2 * M, H = M / 2, LD = H + 1;
    static constexpr int TEAMS = THREADS / T;
    static constexpr int kEx = N;                                    // after the twiddles
    static constexpr int kTwt = kEx + TEAMS * Exch<T, V>::kStride;   // team twiddles
    static constexpr int kB = ((kTwt + team_twiddles<T, V>() + 1) / 2) * 2;
    static constexpr int kTotal = kB + M * LD;                       // float2
};

// Output fields and band limits of the items, passed by value (no host-to-device
// table copy, so a call can be captured in a CUDA graph).  rmax carries the
// item's mirror code in its bits 16+ (yz_mirror).
struct YZOut {
    float *out[CNPC_MAX_ITEMS];
    int rmax[CNPC_MAX_ITEMS];
    int r2max[CNPC_MAX_ITEMS];
};

// A shell of the unit spectrum (source 2) is conj(Y_lm) times a shell mask:
// S(-k) = (-1)^l S(k), so its field has the parity F(-x) = (-1)^l F(x) on the
// grid.  The y/z passes then compute only the planes x <= N/2 and write plane
// N - x as the reflection of plane x (y -> -y, z -> -z mod N, times the sign).
// Code 0: no mirror (data spectra), 1: even (sign +1), 2: odd (sign -1).
__device__ __forceinline__ int yz_rmax(const YZOut &O, int item) { return O.rmax[item] & 0xFFFF; }
__device__ __forceinline__ int yz_mirror(const YZOut &O, int item) { return O.rmax[item] >> 16; }

// Reflected copy of a row with 16-byte stores.  Thread t of a team holds the
// run r(z0 .. z0 + Q2 - 1) of a row, z0 = Q2 t + Q2 T k2 (Q2 T = 2V).  Element z
// goes to (N - z) mod N of the mirror row, so the aligned run at N - z0 - Q2
// is {r(z0 + Q2), r(z0 + Q2 - 1), ..., r(z0 + 1)}: the first value of the next
// run (team lane t + 1 at this k2; for the last lane, lane 0 at k2 + 1, which
// the caller's loop over k2 downwards passes in `carry`) and this run
// reversed.  The run that would need r(N) = r(0) (last lane, k2 = T - 1)
// leaves mirror position 0, which is r(0) itself, to lane 0 after the loop.
template <int T, int Q2>
__device__ __forceinline__ void store_reflected(float *row, int t, int k2, const float *v, float &carry, float sgn,
                                                unsigned mask, int N) {
    float nxt = __shfl_down_sync(mask, v[0], 1, T);
    if (t == T - 1) nxt = carry;
    carry = __shfl_sync(mask, v[0], 0, T);
    const int base = N - (Q2 * t + Q2 * T * k2) - Q2;  // a multiple of 4
    float m[Q2];
    m[0] = sgn * nxt;
#pragma unroll
    for (int c = 1; c < Q2; ++c) m[c] = sgn * v[Q2 - c];
    if (t == T - 1 && k2 == T - 1) {
#pragma unroll
        for (int c = 1; c < Q2; ++c) row[base + c] = m[c];
    } else {
#pragma unroll
        for (int c = 0; c < Q2; c += 4)
            *reinterpret_cast<float4 *>(row + base + c) = make_float4(m[c], m[c + 1], m[c + 2], m[c + 3]);
    }
}

template <int T, int V>
__global__ void __launch_bounds__(YZLayout<T, V>::THREADS, YZLayout<T, V>::MIN_BLOCKS)
    shell_yz_kernel(const float2 *__restrict__ work, int nitems, const YZOut O) {
    using YL = YZLayout<T, V>;
    constexpr int M = YL::M, N = YL::N, H = YL::H, LD = YL::LD, TEAMS = YL::TEAMS;
    constexpr int Q = V / T;
    extern __shared__ float4 smem4[];
    float2 *tw = reinterpret_cast<float2 *>(smem4);
    float2 *Bh = tw + YL::kB;  // [M][LD]: rows y = 2m + ry
    const int item = blockIdx.x % nitems;
    const int ry = (blockIdx.x / nitems) & 1;
    const int x = blockIdx.x / (2 * nitems);
    const int mcode = yz_mirror(O, item);
    if (mcode && x > N / 2) return;  // written by the block of plane N - x
    const bool mirror = mcode && x > 0 && x < N / 2;
    const float msign = mcode == 2 ? -1.f : 1.f;
    float2 *twt = tw + YL::kTwt;
    fill_twiddles(tw, N);
    __syncthreads();
    fill_team_twiddles<T, V>(twt, tw);
    __syncthreads();
    const int team = threadIdx.x / T, t = threadIdx.x % T;
    const unsigned mask = team_mask(T);
    float2 *tex = tw + YL::kEx + team * Exch<T, V>::kStride;
    const float2 *a = work + ((size_t)item * N + x) * M * H;  // A[x][slot][kz]
    const int rmax = yz_rmax(O, item), r2max = O.r2max[item];
    const int K = rmax + 1 < H ? rmax + 1 : H;  // columns k_z >= K are zero
    constexpr int KC = (kKC < H) ? kKC : H;
    // y: one team per k_z column
    for (int kz = team; kz < K; kz += TEAMS) {
        const int kz0 = (kz / KC) * KC;
        float2 u[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const int slot = T * j + t;
            float2 v = make_float2(0.f, 0.f);
            if (slot > 0 && tile_live(slot - H, kz0, r2max)) v = __ldg(a + (size_t)slot * H + kz);
            if (ry) v = cmul(v, tw[slot]);
            u[j] = v;
        }
        team_fft<T, V>(u, t, tex, twt, mask);
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) {
                const int m = team_out_index<T, V>(t, q, k2);
                Bh[m * LD + kz] = shift_phase(u[q * T + k2], m, ry);
            }
    }
    __syncthreads();
    float *fout = O.out[item] + (size_t)x * N * N;
    float *fmir = O.out[item] + (size_t)(N - x) * N * N;  // used when mirror
    // z: row pairs (m1, m2) = (2 p, 2 p + 1) of this parity.  V = 16: teams of
    // one warp take pairs 4 apart, so their rows sit 8 * LD float2 (16 banks)
    // apart.  V = 24 (teams of 4, LD = 49): the 4 teams of a half-warp take
    // pairs 2 apart, rows 4 * LD float2 (8 banks) apart.
    for (int p0 = 0; p0 < M / 2; p0 += TEAMS) {
        const int p = p0 + (V == 24 ? (2 * (team & 3) + ((team >> 2) & 1) + 8 * (team >> 3))
                            : (TEAMS >= 16 && (TEAMS & 15) == 0)
                                ? ((team & 3) * 4 + ((team >> 2) & 3) + 16 * (team >> 4))
                                : team);
        if (p >= M / 2) continue;
        const float2 *b1 = Bh + (2 * p) * LD, *b2 = b1 + LD;
        float2 v[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const int slot = T * j + t;
            const int kz = slot - H;
            const int ak = kz < 0 ? -kz : kz;
            float2 w = make_float2(0.f, 0.f);  // slot 0 (k_z = -n/4) and |k_z| >= K are zero
            if (slot > 0 && ak < K) {
                const float2 c1 = b1[ak], c2 = b2[ak];
                if (kz > 0)
                    w = make_float2(c1.x - c2.y, c1.y + c2.x);
                else if (kz < 0)
                    w = make_float2(c1.x + c2.y, c2.x - c1.y);
                else
                    w = make_float2(c1.x, c2.x);
            }
            v[j] = w;
        }
        float2 res[2][V];
#pragma unroll
        for (int rz = 0; rz < 2; ++rz) {
            float2 u[V];
#pragma unroll
            for (int j = 0; j < V; ++j) u[j] = rz ? cmul(v[j], tw[T * j + t]) : v[j];
            team_fft<T, V>(u, t, tex, twt, mask);
#pragma unroll
            for (int i = 0; i < V; ++i) res[rz][i] = u[i];
        }
        const int y1 = 2 * (2 * p) + ry, y2 = 2 * (2 * p + 1) + ry;  // y = 2 m + ry
        float *row1 = fout + (size_t)y1 * N;
        float *row2 = fout + (size_t)y2 * N;
        float *mrow1 = fmir + (size_t)((N - y1) % N) * N;
        float *mrow2 = fmir + (size_t)((N - y2) % N) * N;
        float carry1 = 0.f, carry2 = 0.f;  // the reflection needs the next (higher) k2's first values
#pragma unroll
        for (int k2 = T - 1; k2 >= 0; --k2) {
            float re[2 * Q], im[2 * Q];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int rz = 0; rz < 2; ++rz) {
                    const int m = team_out_index<T, V>(t, q, k2);
                    const float2 g = shift_phase(res[rz][q * T + k2], m, rz);
                    re[2 * q + rz] = g.x;
                    im[2 * q + rz] = g.y;
                }
            const int z0 = 2 * Q * t + 2 * V * k2;
#pragma unroll
            for (int c = 0; c < 2 * Q; c += 4) {
                *reinterpret_cast<float4 *>(row1 + z0 + c) = make_float4(re[c], re[c + 1], re[c + 2], re[c + 3]);
                *reinterpret_cast<float4 *>(row2 + z0 + c) = make_float4(im[c], im[c + 1], im[c + 2], im[c + 3]);
            }
            if (mirror) {
                store_reflected<T, 2 * Q>(mrow1, t, k2, re, carry1, msign, mask, N);
                store_reflected<T, 2 * Q>(mrow2, t, k2, im, carry2, msign, mask, N);
                if (k2 == 0 && t == 0) {  // mirror position 0 is r(0) itself
                    mrow1[0] = msign * re[0];
                    mrow2[0] = msign * im[0];
                }
            }
        }
    }
}

// Pipelined y/z passes (n = 128): a persistent block walks the (x, y
// parity, item) units of the call with two warp groups that run concurrently
// on two shared buffers.  The y group (YW warps) fills B[j % 2] for unit j
// while the z group (ZW warps) turns B[(j - 1) % 2] into field rows; named
// barriers hand each buffer over (y: arrive "full", z: wait "full"; z: arrive
// "empty", y: wait "empty" before refilling), so the block never waits for all
// its warps at once and the twiddle tables are built once per block.  The
// y pass is one team FFT per k_z column, the z pass two per row pair, so the
// groups are sized to finish a unit together.  The arithmetic and the output
// order of every value are those of shell_yz_kernel.  Timed with CUDA events
// (shell_fields calls of 20 fields): 0.121 -> 0.100 ms at n = 128; at n = 256
// (T = 8, YW = 4 and ZW = 8 or 12, one 133 KB double buffer per SM) it was
// 0.57 -> 0.61 ms, so n = 256 keeps the one-block-per-unit kernel.
template <int T> struct YZPipe {
    static constexpr int YW = T == 8 ? 4 : 2, ZW = T == 8 ? 12 : 4;
    static constexpr int THREADS = 32 * (YW + ZW);
    static constexpr int M = 16 * T, N = 2 * M, H = M / 2, LD = H + 1;
    static constexpr int YT = 32 * YW / T, ZT = 32 * ZW / T;  // teams per group
    static constexpr int kEx = N;
    static constexpr int kTwt = kEx + (YT + ZT) * Exch<T>::kStride;
    static constexpr int kB = ((kTwt + team_twiddles<T>() + 1) / 2) * 2;
    static constexpr int kTotal = kB + 2 * M * LD;  // float2
};

__device__ __forceinline__ void named_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_arrive(int id, int count) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

template <int T>
__global__ void __launch_bounds__(YZPipe<T>::THREADS, 1) shell_yz_pipe_kernel(const float2 *__restrict__ work,
                                                                               int nitems, const YZOut O) {
    using YP = YZPipe<T>;
    constexpr int M = YP::M, N = YP::N, H = YP::H, LD = YP::LD, NT = YP::THREADS;
    constexpr int Q = 16 / T;
    constexpr int KC = (kKC < H) ? kKC : H;
    extern __shared__ float4 smem4[];
    float2 *tw = reinterpret_cast<float2 *>(smem4);
    float2 *twt = tw + YP::kTwt;
    float2 *Bbuf = tw + YP::kB;  // [2][M][LD]
    fill_twiddles(tw, N);
    __syncthreads();
    fill_team_twiddles<T>(twt, tw);
    __syncthreads();
    const int nunits = N * 2 * nitems;
    const int nj = blockIdx.x < nunits ? (nunits - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int warp = threadIdx.x >> 5;
    const int team = threadIdx.x / T, t = threadIdx.x % T;
    const unsigned mask = team_mask(T);
    float2 *tex = tw + YP::kEx + team * Exch<T>::kStride;
    if (warp < YP::YW) {
        // ------------------------------------------------ y pass (producer)
        for (int j = 0; j < nj; ++j) {
            const int u = blockIdx.x + j * gridDim.x;
            const int item = u % nitems, ry = (u / nitems) & 1, x = u / (2 * nitems);
            const int b = j & 1;
            if (j >= 2) named_sync(3 + b, NT);  // the z group has drained this buffer
            float2 *Bh = Bbuf + b * M * LD;
            const float2 *a = work + ((size_t)item * N + x) * M * H;
            const int rmax = yz_rmax(O, item), r2max = O.r2max[item];
            // a mirrored item's planes x > N/2 are written by plane N - x: the
            // unit keeps its barrier steps and does no work
            const bool skip = yz_mirror(O, item) && x > N / 2;
            const int K = skip ? 0 : (rmax + 1 < H ? rmax + 1 : H);
            for (int kz = team; kz < K; kz += YP::YT) {
                const int kz0 = (kz / KC) * KC;
                float2 u16[16];
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {
                    const int slot = T * jj + t;
                    float2 v = make_float2(0.f, 0.f);
                    if (slot > 0 && tile_live(slot - H, kz0, r2max)) v = __ldg(a + (size_t)slot * H + kz);
                    if (ry) v = cmul(v, tw[slot]);
                    u16[jj] = v;
                }
                team_fft<T>(u16, t, tex, twt, mask);
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int k2 = 0; k2 < T; ++k2) {
                        const int m = team_out_index<T>(t, q, k2);
                        Bh[m * LD + kz] = shift_phase(u16[q * T + k2], m, ry);
                    }
            }
            named_arrive(1 + b, NT);
        }
    } else {
        // ------------------------------------------------ z pass (consumer)
        const int zteam = team - YP::YT;
        for (int j = 0; j < nj; ++j) {
            const int u = blockIdx.x + j * gridDim.x;
            const int item = u % nitems, ry = (u / nitems) & 1, x = u / (2 * nitems);
            const int b = j & 1;
            named_sync(1 + b, NT);  // the y group has filled this buffer
            const float2 *Bh = Bbuf + b * M * LD;
            const int rmax = yz_rmax(O, item);
            const int K = rmax + 1 < H ? rmax + 1 : H;
            const int mcode = yz_mirror(O, item);
            const bool skip = mcode && x > N / 2;  // same test as the y group
            const bool mirror = mcode && x > 0 && x < N / 2;
            const float msign = mcode == 2 ? -1.f : 1.f;
            float *fout = O.out[item] + (size_t)x * N * N;
            float *fmir = O.out[item] + (size_t)(N - x) * N * N;
            for (int p0 = 0; p0 < (skip ? 0 : M / 2); p0 += YP::ZT) {
                // teams of one warp take pairs 4 apart (rows 8 LD float2 apart)
                const int p = p0 + ((zteam & 3) * 4 + ((zteam >> 2) & 3) + 16 * (zteam >> 4));
                if (p >= M / 2) continue;
                const float2 *b1 = Bh + (2 * p) * LD, *b2 = b1 + LD;
                float2 v[16];
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {
                    const int slot = T * jj + t;
                    const int kz = slot - H;
                    const int ak = kz < 0 ? -kz : kz;
                    float2 w = make_float2(0.f, 0.f);
                    if (slot > 0 && ak < K) {
                        const float2 c1 = b1[ak], c2 = b2[ak];
                        if (kz > 0)
                            w = make_float2(c1.x - c2.y, c1.y + c2.x);
                        else if (kz < 0)
                            w = make_float2(c1.x + c2.y, c2.x - c1.y);
                        else
                            w = make_float2(c1.x, c2.x);
                    }
                    v[jj] = w;
                }
                float2 res[2][16];
#pragma unroll
                for (int rz = 0; rz < 2; ++rz) {
                    float2 u16[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) u16[jj] = rz ? cmul(v[jj], tw[T * jj + t]) : v[jj];
                    team_fft<T>(u16, t, tex, twt, mask);
#pragma unroll
                    for (int i = 0; i < 16; ++i) res[rz][i] = u16[i];
                }
                const int y1 = 2 * (2 * p) + ry, y2 = 2 * (2 * p + 1) + ry;
                float *row1 = fout + (size_t)y1 * N;
                float *row2 = fout + (size_t)y2 * N;
                float *mrow1 = fmir + (size_t)((N - y1) & (N - 1)) * N;
                float *mrow2 = fmir + (size_t)((N - y2) & (N - 1)) * N;
                float carry1 = 0.f, carry2 = 0.f;
#pragma unroll
                for (int k2 = T - 1; k2 >= 0; --k2) {
                    float re[2 * Q], im[2 * Q];
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int rz = 0; rz < 2; ++rz) {
                            const int m = team_out_index<T>(t, q, k2);
                            const float2 g = shift_phase(res[rz][q * T + k2], m, rz);
                            re[2 * q + rz] = g.x;
                            im[2 * q + rz] = g.y;
                        }
                    const int z0 = 2 * Q * t + 32 * k2;
#pragma unroll
                    for (int c = 0; c < 2 * Q; c += 4) {
                        *reinterpret_cast<float4 *>(row1 + z0 + c) = make_float4(re[c], re[c + 1], re[c + 2], re[c + 3]);
                        *reinterpret_cast<float4 *>(row2 + z0 + c) = make_float4(im[c], im[c + 1], im[c + 2], im[c + 3]);
                    }
                    if (mirror) {
                        store_reflected<T, 2 * Q>(mrow1, t, k2, re, carry1, msign, mask, N);
                        store_reflected<T, 2 * Q>(mrow2, t, k2, im, carry2, msign, mask, N);
                        if (k2 == 0 && t == 0) {
                            mrow1[0] = msign * re[0];
                            mrow2[0] = msign * im[0];
                        }
                    }
                }
            }
            if (j + 2 < nj) named_arrive(3 + b, NT);  // the y group refills it for unit j + 2
        }
    }
}

// ------------------------------------------------------------ dispatch
// the pipelined y/z kernel for n = 128 (false: one block per unit)
constexpr bool kShellPipeline = true;

template <int T, int V> static size_t column_smem(int nedges) {
    const int M = V * T, N = 2 * M, H = M / 2, KC = kKC < H ? kKC : H, LDC = KC + 1;
    return sizeof(float2) * ((size_t)M * LDC + (size_t)N * LDC + N + (kColThreads / T) * Exch<T, V>::kStride +
                             team_twiddles<T, V>()) +
           sizeof(double) * (N + 1 + nedges);
}
template <int T, int V> static size_t yz_smem() { return sizeof(float2) * (size_t)YZLayout<T, V>::kTotal; }

template <int T, int V>
static int launch_shell_fft(cnpc_ctx *ctx, int n, double L, const float2 *A, const float2 *B, const EdgeSet &es,
                            const HarmTable &ht, const ShellItemsDev &items, float2 *workA,
                            const YZOut &O, cudaStream_t s) {
    constexpr int M = V * T, N = 2 * M, H = M / 2;
    constexpr int KC = kKC < H ? kKC : H;
    constexpr int NCH = H / KC;
    static_assert(H % KC == 0, "column chunks must tile n/4");
    const size_t sc = column_smem<T, V>(es.n), sr = yz_smem<T, V>();
    int st = check_cuda(ctx, cudaFuncSetAttribute(shell_column_kernel<T, V>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sc), "shell smem");
    if (st) return st;
    st = check_cuda(ctx, cudaFuncSetAttribute(shell_yz_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)sr), "shell smem");
    if (st) return st;
    const int ni = items.n;
    shell_column_kernel<T, V><<<(M - 1) * NCH * ni, kColThreads, sc, s>>>(A, B, n, L, es, ht, items, workA);
    if constexpr (T == 4 && V == 16 && kShellPipeline) {
        using YP = YZPipe<T>;
        const size_t sp = sizeof(float2) * (size_t)YP::kTotal;
        st = check_cuda(ctx, cudaFuncSetAttribute(shell_yz_pipe_kernel<T>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp),
                        "shell smem");
        if (st) return st;
        int per_sm = 1;
        st = check_cuda(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, shell_yz_pipe_kernel<T>,
                                                                           YP::THREADS, sp), "shell occupancy");
        if (st) return st;
        const int grid = std::min(N * 2 * ni, std::max(1, per_sm) * ctx->num_sms);
        shell_yz_pipe_kernel<T><<<grid, YP::THREADS, sp, s>>>(workA, ni, O);
    } else {
        shell_yz_kernel<T, V><<<N * 2 * ni, YZLayout<T, V>::THREADS, sr, s>>>(workA, ni, O);
    }
    return check_launch(ctx, "shell_fields kernels");
}

// out[x][y][z] for the planes x = 0 .. n/2: in[x][y][z] on the planes 0 and
// n/2, in[x][y][z] + sign in[n - x][-y][-z] (indices mod n) on the others.
template <typename T>
__global__ void parity_fold_kernel(const T *__restrict__ in, T *__restrict__ out, int n, T sign) {
    const int64_t nn = (int64_t)n * n;
    const int64_t total = (int64_t)(n / 2 + 1) * nn;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i / nn);
        const int y = (int)((i / n) % n), z = (int)(i % n);
        T v = in[i];
        if (x > 0 && x < n / 2) {
            const int yr = y == 0 ? 0 : n - y, zr = z == 0 ? 0 : n - z;
            v += sign * in[((int64_t)(n - x) * n + yr) * n + zr];
        }
        out[i] = v;
    }
}

// FP32 form of parity_fold_kernel for n % 4 == 0: one warp per row (x, y),
// 16-byte loads and stores.  Element z of the row needs the mirror row's
// element (n - z) mod n; for the float4 j (z = 4j .. 4j + 3) those are
// p.w, p.z, p.y of the mirror row's float4 n/4 - 1 - j and, first, the
// element n - 4j, which is the x of the float4 the lane before loads (lane 0
// reads it directly).  Same sums, same rounding as parity_fold_kernel.
__global__ void parity_fold_rows_kernel(const float *__restrict__ in, float *__restrict__ out, int n, float sign) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int nrows = (n / 2 + 1) * n, nq = n / 4;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows; r += warps) {
        const int x = r / n, y = r % n;
        const float4 *src = reinterpret_cast<const float4 *>(in + (size_t)r * n);
        float4 *dst = reinterpret_cast<float4 *>(out + (size_t)r * n);
        if (x == 0 || x == n / 2) {
            for (int j = lane; j < nq; j += 32) dst[j] = src[j];
            continue;
        }
        const int yr = y == 0 ? 0 : n - y;
        const float *mrow = in + ((size_t)(n - x) * n + yr) * n;
        const float4 *m4 = reinterpret_cast<const float4 *>(mrow);
        for (int j0 = 0; j0 < nq; j0 += 32) {
            const int j = j0 + lane;
            const bool ok = j < nq;
            const float4 p = ok ? m4[nq - 1 - j] : make_float4(0.f, 0.f, 0.f, 0.f);
            float first = __shfl_up_sync(0xffffffffu, p.x, 1);
            if (lane == 0) first = mrow[(n - 4 * j) % n];
            if (ok) {
                float4 v = src[j];
                v.x += sign * first;
                v.y += sign * p.w;
                v.z += sign * p.z;
                v.w += sign * p.y;
                dst[j] = v;
            }
        }
    }
}

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_field_parity_fold(cnpc_ctx *ctx, int dtype, int n, const void *d_in, int sign, void *d_out,
                                      cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    CNPC_REQUIRE(ctx, n >= 2 && n % 2 == 0 && n <= 2048, "n must be even, 2..2048");
    CNPC_REQUIRE(ctx, sign == 1 || sign == -1, "sign must be +1 or -1");
    CNPC_REQUIRE(ctx, d_in && d_out && d_in != d_out, "null or aliased buffer");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t total = (int64_t)(n / 2 + 1) * n * n;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 8);
    const bool rows16 = n % 4 == 0 && reinterpret_cast<uintptr_t>(d_in) % 16 == 0 &&
                        reinterpret_cast<uintptr_t>(d_out) % 16 == 0;
    if (dtype == CNPC_F32 && rows16) {
        // one warp per row, 8 warps per block
        const int64_t rows = (int64_t)(n / 2 + 1) * n;
        const int rblocks = (int)std::min<int64_t>((rows + 7) / 8, (int64_t)ctx->num_sms * 8);
        parity_fold_rows_kernel<<<rblocks, 256, 0, s>>>((const float *)d_in, (float *)d_out, n, (float)sign);
    } else if (dtype == CNPC_F32)
        parity_fold_kernel<float><<<blocks, 256, 0, s>>>((const float *)d_in, (float *)d_out, n, (float)sign);
    else
        parity_fold_kernel<double><<<blocks, 256, 0, s>>>((const double *)d_in, (double *)d_out, n, (double)sign);
    return check_launch(ctx, "parity_fold_kernel");
}

extern "C" int cnpc_shell_fields(cnpc_ctx *ctx, int n, double boxsize, const void *d_spec_a, const void *d_spec_b,
                                 const double *h_edges, int nedges, const cnpc_harmonic *h_harmonics,
                                 int nharmonics, const cnpc_shell_item *h_items, int nitems,
                                 void *const *h_out_fields, cnpc_stream_t stream) {
    int st = check_common(ctx, CNPC_F32, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, n == 64 || n == 128 || n == 192 || n == 256, "fused shell fields support n = 64, 128, 192, 256");
    CNPC_REQUIRE(ctx, nitems >= 1 && nitems <= CNPC_MAX_ITEMS, "nitems out of range (1..256)");
    CNPC_REQUIRE(ctx, nharmonics >= 1 && nharmonics <= CNPC_MAX_HARMONICS, "nharmonics out of range");
    CNPC_REQUIRE(ctx, h_harmonics && h_items && h_out_fields, "null table");
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
    ShellItemsDev items;
    items.n = nitems;
    const double kf = 2.0 * kPi / boxsize;
    for (int j = 0; j < nitems; ++j) {
        const cnpc_shell_item &it = h_items[j];
        CNPC_REQUIRE(ctx, it.bin >= 0 && it.bin < nedges - 1, "item bin out of range");
        CNPC_REQUIRE(ctx, it.harmonic >= 0 && it.harmonic < nharmonics, "item harmonic out of range");
        CNPC_REQUIRE(ctx, it.component == 0 || it.component == 1, "item component must be 0/1");
        CNPC_REQUIRE(ctx, it.source >= 0 && it.source <= 2, "item source must be 0..2");
        CNPC_REQUIRE(ctx, it.source != 0 || d_spec_a, "item needs spectrum A");
        CNPC_REQUIRE(ctx, it.source != 1 || d_spec_b, "item needs spectrum B");
        CNPC_REQUIRE(ctx, h_out_fields[j] != nullptr, "null output field");
        CNPC_REQUIRE(ctx, reinterpret_cast<uintptr_t>(h_out_fields[j]) % 16 == 0, "output fields must be 16-byte aligned");
        // every mode of the shell must lie in |n_d| < n/4
        CNPC_REQUIRE(ctx, h_edges[it.bin + 1] / kf < n / 4.0, "shell band reaches n/4 (needs k < k_Nyquist / 2)");
        items.it[j] = it;
        const double rt = h_edges[it.bin + 1] / kf * (1.0 + 1e-9);
        items.rmax[j] = (int)std::floor(rt);
        items.r2max[j] = (int)std::floor(rt * rt) + 1;
    }
    const size_t per_item_a = sizeof(float2) * (size_t)n * (n / 2) * (n / 4);  // A[x][s][n_z]
    cudaStream_t s = (cudaStream_t)stream;
    // the pass-1 work array
    st = ensure_buffer(ctx, &ctx->shell_ws, &ctx->shell_ws_bytes, per_item_a * nitems, s);
    if (st) return st;
    float2 *workA = static_cast<float2 *>(ctx->shell_ws);
    YZOut O;
    std::memset(&O, 0, sizeof(O));
    for (int j = 0; j < nitems; ++j) {
        O.out[j] = static_cast<float *>(h_out_fields[j]);
        // unit-spectrum shells have the parity (-1)^l: mirror code in bits 16+
        const int mcode = kMirrorUnitShells && items.it[j].source == 2 ? ((ht.h[items.it[j].harmonic].l & 1) ? 2 : 1) : 0;
        O.rmax[j] = items.rmax[j] | (mcode << 16);
        O.r2max[j] = items.r2max[j];
    }
    const float2 *A = static_cast<const float2 *>(d_spec_a);
    const float2 *B = static_cast<const float2 *>(d_spec_b);
    if (n == 64) return launch_shell_fft<2, 16>(ctx, n, boxsize, A, B, es, ht, items, workA, O, s);
    if (n == 128) return launch_shell_fft<4, 16>(ctx, n, boxsize, A, B, es, ht, items, workA, O, s);
    if (n == 192) return launch_shell_fft<4, 24>(ctx, n, boxsize, A, B, es, ht, items, workA, O, s);
    return launch_shell_fft<8, 16>(ctx, n, boxsize, A, B, es, ht, items, workA, O, s);
}
