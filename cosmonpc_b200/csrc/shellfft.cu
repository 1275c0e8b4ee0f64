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
// The n/2-point FFT is done by a team of T = n/32 threads holding 16 values
// each: a 16-point DFT in registers, twiddles, one shared-memory exchange and
// T-point DFTs.  Twiddles come from an FP64-computed table rounded to FP32.
#include <cmath>
#include <vector>

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

// Team FFT of size M = 16 T (inverse).  On entry thread t of the team holds
// u[j] = x[T j + t]; on exit it holds X[k1 + 16 k2] for k1 = t (16/T) + q
// (q < 16/T), k2 < T, stored as u[q * T + k2].  ex: the team's 16 T exchange
// slots; tw: W_n table (n = 2M entries; W_M^j = tw[2 j]).
template <int T>
__device__ __forceinline__ void team_fft(float2 *u, int t, float2 *ex, const float2 *tw, unsigned mask) {
    idft16(u);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) u[k1] = cmul(u[k1], tw[2 * ((t * k1) % (16 * T))]);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) ex[k1 * T + t] = u[k1];
    __syncwarp(mask);
    constexpr int Q = 16 / T;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int k1 = t * Q + q;
        float2 w[T];
#pragma unroll
        for (int i = 0; i < T; ++i) w[i] = ex[k1 * T + i];
        if (T == 2) idft2(w[0], w[1]);
        if (T == 4) idft4(w[0], w[1], w[2], w[3]);
        if (T == 8) idft8(w);
#pragma unroll
        for (int i = 0; i < T; ++i) u[q * T + i] = w[i];
    }
    __syncwarp(mask);
}

// output index m (of the M-point transform) held in u[q T + k2]
template <int T>
__device__ __forceinline__ int team_out_index(int t, int q, int k2) {
    return (t * (16 / T) + q) + 16 * k2;
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
};

}  // namespace

// ---------------------------------------------------------------- pass 1
// One block per (row slot s = n_y + n/4 in [1, n/2), item).  Synthesises the
// item's columns (all n_x, n_z in band) from the source spectrum, transforms
// them along x and writes A_item[x][s][n_z].
template <int T>
__global__ void __launch_bounds__(128) shell_xpass_kernel(const float2 *__restrict__ A, const float2 *__restrict__ B,
                                                          int n, double L, EdgeSet edges, HarmTable harm,
                                                          ShellItemsDev items, float2 *__restrict__ work) {
    constexpr int M = 16 * T;   // n / 2
    constexpr int N = 2 * M;    // n
    constexpr int H = M / 2;    // n / 4: band half-width (slots) and n_z count
    constexpr int LD = H + 1;   // padded row of n_z values
    extern __shared__ float4 smem4[];
    float2 *in = reinterpret_cast<float2 *>(smem4);  // [M slots][LD]
    float2 *out = in + M * LD;                       // [N x][LD]
    float2 *tw = out + N * LD;                       // [N] twiddles W_n^j
    float2 *ex = tw + N;                             // [teams][16 T]
    double *kt = reinterpret_cast<double *>(ex + (blockDim.x / T) * 16 * T);  // [n + 1] k table
    const int s = 1 + blockIdx.x / items.n;
    const int item = blockIdx.x % items.n;
    const cnpc_shell_item it = items.it[item];
    const cnpc_harmonic &hm = harm.h[it.harmonic];
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * j / N, &sn, &cs);
        tw[j] = make_float2((float)cs, (float)sn);
    }
    for (int i = threadIdx.x; i <= n; i += blockDim.x) kt[i] = kcomp(i - n / 2, L);
    __syncthreads();
    const int ny = s - H;
    const int iy = ny < 0 ? ny + n : ny;
    const int nh2 = n / 2 + 1;
    // synthesise the (n_x slot, n_z) tile of this row
    for (int e = threadIdx.x; e < M * H; e += blockDim.x) {
        const int xs = e / H, nz = e % H;
        float2 v = make_float2(0.f, 0.f);
        if (xs > 0) {
            const int nx = xs - H;
            const int ix = nx < 0 ? nx + n : nx;
            const double kx = kt[nx + n / 2], ky = kt[ny + n / 2], kz = kt[nz + n / 2];
            const double kn = knorm_from(kx, ky, kz);
            if (find_bin(kn, edges.e, edges.n) == it.bin) {
                const bool origin = kn == 0.0;
                const double ik = origin ? 0.0 : 1.0 / kn;
                float2 Y = harmonic_eval<float>(hm, (float)(kx * ik), (float)(ky * ik), (float)(kz * ik), origin);
                if (it.conj) Y.y = -Y.y;
                float2 phi;
                if ((hm.l & 1) == 0)
                    phi = it.component == 0 ? make_float2(Y.x, 0.f) : make_float2(Y.y, 0.f);
                else
                    phi = it.component == 0 ? make_float2(0.f, Y.y) : make_float2(0.f, -Y.x);
                float2 src;
                const int64_t t = ((int64_t)ix * n + iy) * nh2 + nz;
                if (it.source == 0)
                    src = A[t];
                else if (it.source == 1)
                    src = B[t];
                else
                    src = make_float2(1.f, 0.f);
                v = cmul(src, phi);
            }
        }
        in[xs * LD + nz] = v;
    }
    __syncthreads();
    // inverse DFT along x of each n_z column, both output parities
    const int team = threadIdx.x / T, t = threadIdx.x % T, nteams = blockDim.x / T;
    const unsigned mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) & ~(T - 1)));
    float2 *tex = ex + team * 16 * T;
    for (int job = team; job < 2 * H; job += nteams) {
        const int nz = job >> 1, r = job & 1;
        float2 u[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int slot = T * j + t;
            float2 v = in[slot * LD + nz];
            if (r) v = cmul(v, tw[slot]);
            u[j] = v;
        }
        team_fft<T>(u, t, tex, tw, mask);
#pragma unroll
        for (int q = 0; q < 16 / T; ++q)
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) {
                const int m = team_out_index<T>(t, q, k2);
                out[(2 * m + r) * LD + nz] = shift_phase(u[q * T + k2], m, r);
            }
    }
    __syncthreads();
    // A_item[x][s][n_z]
    float2 *dst = work + (size_t)item * N * M * H;
    for (int e = threadIdx.x; e < N * H; e += blockDim.x) {
        const int x = e / H, nz = e % H;
        dst[((size_t)x * M + s) * H + nz] = out[x * LD + nz];
    }
}

// ---------------------------------------------------------------- pass 2
constexpr int kShellThreads = 128;
// two staged output rows of N = 32 T floats per team of T threads: 64 kShellThreads floats
constexpr int kStagedFloat2 = 32 * kShellThreads;
// One block per (x, item): y-transform of the n/4 columns, then the real
// z-output two rows at a time; writes field[x][y][z].
template <int T>
__global__ void __launch_bounds__(kShellThreads) shell_yzpass_kernel(const float2 *__restrict__ work, int nitems,
                                                           float *const *__restrict__ outs) {
    constexpr int M = 16 * T;
    constexpr int N = 2 * M;
    constexpr int H = M / 2;
    constexpr int LD = H + 1;
    // A region: the [M slots][LD] input, later the teams' staged output rows
    constexpr int ASZ = (M * LD > kStagedFloat2) ? M * LD : kStagedFloat2;
    extern __shared__ float4 smem4[];
    float2 *A = reinterpret_cast<float2 *>(smem4);
    float2 *B = A + ASZ;                            // [N y][LD]
    float2 *tw = B + N * LD;                        // [N]
    float2 *ex = tw + N;                            // [teams][16 T]
    const int x = blockIdx.x / nitems;
    const int item = blockIdx.x % nitems;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * j / N, &sn, &cs);
        tw[j] = make_float2((float)cs, (float)sn);
    }
    const float2 *src = work + ((size_t)item * N + x) * M * H;
    for (int e = threadIdx.x; e < M * H; e += blockDim.x) {
        const int s = e / H, nz = e % H;
        A[s * LD + nz] = s == 0 ? make_float2(0.f, 0.f) : src[e];
    }
    __syncthreads();
    const int team = threadIdx.x / T, t = threadIdx.x % T, nteams = blockDim.x / T;
    const unsigned mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) & ~(T - 1)));
    float2 *tex = ex + team * 16 * T;
    // y: B[y][n_z]
    for (int job = team; job < 2 * H; job += nteams) {
        const int nz = job >> 1, r = job & 1;
        float2 u[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int slot = T * j + t;
            float2 v = A[slot * LD + nz];
            if (r) v = cmul(v, tw[slot]);
            u[j] = v;
        }
        team_fft<T>(u, t, tex, tw, mask);
#pragma unroll
        for (int q = 0; q < 16 / T; ++q)
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) {
                const int m = team_out_index<T>(t, q, k2);
                B[(2 * m + r) * LD + nz] = shift_phase(u[q * T + k2], m, r);
            }
    }
    __syncthreads();
    // z: rows y1 = 2p, y2 = 2p + 1 through one complex transform of
    // v(k_z) = B1~(k_z) + i B2~(k_z), B~(-k_z) = conj B(k_z), B~(0) = Re B(0)
    float *rows = reinterpret_cast<float *>(A) + team * 2 * N;  // two staged rows per team
    float *dst = outs[item] + (size_t)x * N * N;
    for (int p = team; p < N / 2; p += nteams) {
        const float2 *b1 = B + (2 * p) * LD, *b2 = B + (2 * p + 1) * LD;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            float2 u[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int slot = T * j + t;
                const int kz = slot - H;
                float2 v = make_float2(0.f, 0.f);  // slot 0 is k_z = -n/4, outside the band
                if (kz > 0)
                    v = make_float2(b1[kz].x - b2[kz].y, b1[kz].y + b2[kz].x);
                else if (kz < 0 && slot > 0)
                    v = make_float2(b1[-kz].x + b2[-kz].y, b2[-kz].x - b1[-kz].y);
                else if (kz == 0)
                    v = make_float2(b1[0].x, b2[0].x);
                if (r) v = cmul(v, tw[slot]);
                u[j] = v;
            }
            team_fft<T>(u, t, tex, tw, mask);
#pragma unroll
            for (int q = 0; q < 16 / T; ++q)
#pragma unroll
                for (int k2 = 0; k2 < T; ++k2) {
                    const int m = team_out_index<T>(t, q, k2);
                    const float2 g = shift_phase(u[q * T + k2], m, r);
                    rows[2 * m + r] = g.x;
                    rows[N + 2 * m + r] = g.y;
                }
        }
        __syncwarp(mask);
        float4 *d1 = reinterpret_cast<float4 *>(dst + (size_t)(2 * p) * N);
        const float4 *s4 = reinterpret_cast<const float4 *>(rows);
        for (int i = t; i < N / 2; i += T) d1[i] = s4[i];  // both rows are contiguous in the field
        __syncwarp(mask);
    }
}

// ------------------------------------------------------------ dispatch
static size_t xpass_smem(int T, int threads) {
    const int M = 16 * T, N = 2 * M, LD = M / 2 + 1;
    return sizeof(float2) * ((size_t)M * LD + (size_t)N * LD + N + (threads / T) * 16 * T) +
           sizeof(double) * (N + 1);
}
static size_t yzpass_smem(int T, int threads) {
    const int M = 16 * T, N = 2 * M, LD = M / 2 + 1;
    size_t a = (size_t)M * LD;
    if ((size_t)kStagedFloat2 > a) a = kStagedFloat2;  // same A region as the kernel
    return sizeof(float2) * (a + (size_t)N * LD + N + (threads / T) * 16 * T);
}

template <int T>
static int launch_shell_fft(cnpc_ctx *ctx, int n, double L, const float2 *A, const float2 *B, const EdgeSet &es,
                            const HarmTable &ht, const ShellItemsDev &items, float2 *work, float *const *d_outs,
                            cudaStream_t s) {
    const int threads = kShellThreads;
    const size_t s1 = xpass_smem(T, threads), s2 = yzpass_smem(T, threads);
    int st = check_cuda(ctx, cudaFuncSetAttribute(shell_xpass_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)s1), "shell xpass smem");
    if (st) return st;
    st = check_cuda(ctx, cudaFuncSetAttribute(shell_yzpass_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)s2), "shell yzpass smem");
    if (st) return st;
    const int M = 16 * T;
    shell_xpass_kernel<T><<<(M - 1) * items.n, threads, s1, s>>>(A, B, n, L, es, ht, items, work);
    st = check_launch(ctx, "shell_xpass_kernel");
    if (st) return st;
    shell_yzpass_kernel<T><<<n * items.n, threads, s2, s>>>(work, items.n, d_outs);
    return check_launch(ctx, "shell_yzpass_kernel");
}

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_shell_fields(cnpc_ctx *ctx, int n, double boxsize, const void *d_spec_a, const void *d_spec_b,
                                 const double *h_edges, int nedges, const cnpc_harmonic *h_harmonics,
                                 int nharmonics, const cnpc_shell_item *h_items, int nitems,
                                 void *const *h_out_fields, cnpc_stream_t stream) {
    int st = check_common(ctx, CNPC_F32, n, boxsize);
    if (st) return st;
    CNPC_REQUIRE(ctx, n == 64 || n == 128 || n == 256, "fused shell fields support n = 64, 128, 256");
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
    }
    const int T = n / 32;
    const size_t per_item = sizeof(float2) * (size_t)n * (n / 2) * (n / 4);
    cudaStream_t s = (cudaStream_t)stream;
    // output pointer table and the pass-1 work array in one workspace
    const size_t ptr_bytes = (sizeof(float *) * nitems + 255) / 256 * 256;
    st = ensure_buffer(ctx, &ctx->shell_ws, &ctx->shell_ws_bytes, ptr_bytes + per_item * nitems, s);
    if (st) return st;
    float **d_ptrs = static_cast<float **>(ctx->shell_ws);
    float2 *work = reinterpret_cast<float2 *>(static_cast<char *>(ctx->shell_ws) + ptr_bytes);
    std::vector<float *> hp(nitems);
    for (int j = 0; j < nitems; ++j) hp[j] = static_cast<float *>(h_out_fields[j]);
    // pageable source: the copy completes before the call returns
    st = check_cuda(ctx, cudaMemcpyAsync(d_ptrs, hp.data(), sizeof(float *) * nitems, cudaMemcpyHostToDevice, s),
                    "shell output table");
    if (st) return st;
    const float2 *A = static_cast<const float2 *>(d_spec_a);
    const float2 *B = static_cast<const float2 *>(d_spec_b);
    if (T == 2) return launch_shell_fft<2>(ctx, n, boxsize, A, B, es, ht, items, work, d_ptrs, s);
    if (T == 4) return launch_shell_fft<4>(ctx, n, boxsize, A, B, es, ht, items, work, d_ptrs, s);
    return launch_shell_fft<8>(ctx, n, boxsize, A, B, es, ht, items, work, d_ptrs, s);
}
