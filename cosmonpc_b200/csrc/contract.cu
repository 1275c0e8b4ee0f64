// x-space triple-product reductions  sum_x G(x) F_a(x) F_b(x).
//
// Gram form: rows a_0..a_{na-1}, columns b_0..b_{nb-1}.  Each warp owns one
// TM x TN output tile; its 32 lanes stride over the cells of a chunk that the
// block stages in shared memory (G plus every field the block's tiles touch).
// FP32 fields: a lane accumulates TM*TN products in FP32 for `flush_chunks`
// chunks, then the warp folds the 32 lane partials with a recursive-halving
// shuffle transpose (lane l ends with tile elements 2l, 2l+1) and adds them
// into FP64 registers.  FP64 fields accumulate in FP64 throughout.  Each block
// writes its FP64 tile partials; a second kernel sums them in a fixed order,
// so results are bitwise reproducible.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace cnpc {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kMaxRows = 128;
constexpr int kMaxUnion = 256;

template <typename T> struct TileShape;
template <> struct TileShape<float> { static constexpr int TM = 8, TN = 8; };
template <> struct TileShape<double> { static constexpr int TM = 8, TN = 4; };

struct GramParams {
    int na, nb, nunion, ct, ntiles, ngroups, chunk, flush_chunks, vec_ok;
    int64_t ncell, field_stride;
    int a_slot[kMaxRows];
    int b_slot[kMaxRows];
    int union_field[kMaxUnion];
};

// Recursive-halving transpose reduction over the 32 lanes of a warp.
template <typename V, int LEN, int S> struct TransposeReduce {
    __device__ static inline void run(V *v, int lane) {
        constexpr int H = LEN / 2;
        const bool hi = (lane & S) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const V keep = hi ? v[i + H] : v[i];
            const V send = hi ? v[i] : v[i + H];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, S);
        }
        TransposeReduce<V, H, S / 2>::run(v, lane);
    }
};
template <typename V, int LEN> struct TransposeReduce<V, LEN, 0> {
    __device__ static inline void run(V *, int) {}
};

template <typename T>
__global__ void __launch_bounds__(kThreads) gram_kernel(const T *__restrict__ g,
                                                        const T *__restrict__ fields,
                                                        const GramParams P, double *partial) {
    constexpr int TM = TileShape<T>::TM, TN = TileShape<T>::TN, NV = TM * TN;
    constexpr int PER_LANE = NV / 32;  // tile elements owned by a lane after the fold
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // staged rows: row 0 is G, row u >= 1 is field union_field[u - 1]
    T *sG = reinterpret_cast<T *>(smem_raw);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int group = blockIdx.x % P.ngroups;
    const int xr = blockIdx.x / P.ngroups;
    const int nxr = gridDim.x / P.ngroups;
    const int tile = group * kWarps + warp;
    const bool active = tile < P.ntiles;
    const int rt = active ? tile / P.ct : 0;
    const int cti = active ? tile % P.ct : 0;

    int rs[TM], cs[TN];
#pragma unroll
    for (int r = 0; r < TM; ++r) {
        const int i = min(rt * TM + r, P.na - 1);
        rs[r] = P.a_slot[i] * P.chunk;
    }
#pragma unroll
    for (int c = 0; c < TN; ++c) {
        const int j = min(cti * TN + c, P.nb - 1);
        cs[c] = P.b_slot[j] * P.chunk;
    }

    T acc[NV];
#pragma unroll
    for (int e = 0; e < NV; ++e) acc[e] = (T)0;
    double acc64[PER_LANE];
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) acc64[e] = 0.0;

    const int nf = P.nunion + 1;  // staged rows: G then the union fields
    const bool vec = P.vec_ok != 0;
    int since_flush = 0;
    for (int64_t c0 = (int64_t)xr * P.chunk; c0 < P.ncell; c0 += (int64_t)nxr * P.chunk) {
        __syncthreads();
        // ---- stage G and the fields of this chunk
        if (vec && c0 + P.chunk <= P.ncell) {
            const int q = P.chunk / 4;
            for (int idx = threadIdx.x; idx < nf * q; idx += kThreads) {
                const int u = idx / q, c4 = (idx % q) * 4;
                const T *src = u == 0 ? g + c0 : fields + (int64_t)P.union_field[u - 1] * P.field_stride + c0;
                T *dst = sG + (int64_t)u * P.chunk + c4;
                if (sizeof(T) == 4) {
                    *reinterpret_cast<float4 *>(dst) = __ldg(reinterpret_cast<const float4 *>(src + c4));
                } else {
                    const double2 *s2 = reinterpret_cast<const double2 *>(src + c4);
                    reinterpret_cast<double2 *>(dst)[0] = __ldg(s2);
                    reinterpret_cast<double2 *>(dst)[1] = __ldg(s2 + 1);
                }
            }
        } else {
            for (int idx = threadIdx.x; idx < nf * P.chunk; idx += kThreads) {
                const int u = idx / P.chunk, c = idx % P.chunk;
                const int64_t cell = c0 + c;
                T v = (T)0;
                if (cell < P.ncell)
                    v = u == 0 ? g[cell] : fields[(int64_t)P.union_field[u - 1] * P.field_stride + cell];
                sG[(int64_t)u * P.chunk + c] = v;
            }
        }
        __syncthreads();
        if (!active) continue;
        // ---- accumulate this warp's tile over the chunk
        for (int c = lane; c < P.chunk; c += 32) {
            const T gv = sG[c];
            T av[TM], bv[TN];
#pragma unroll
            for (int r = 0; r < TM; ++r) av[r] = gv * sG[rs[r] + c];
#pragma unroll
            for (int s = 0; s < TN; ++s) bv[s] = sG[cs[s] + c];
#pragma unroll
            for (int r = 0; r < TM; ++r)
#pragma unroll
                for (int s = 0; s < TN; ++s) acc[r * TN + s] += av[r] * bv[s];
        }
        if (sizeof(T) == 4 && ++since_flush == P.flush_chunks) {
            since_flush = 0;
            TransposeReduce<T, NV, 16>::run(acc, lane);
#pragma unroll
            for (int e = 0; e < PER_LANE; ++e) acc64[e] += (double)acc[e];
#pragma unroll
            for (int e = 0; e < NV; ++e) acc[e] = (T)0;
        }
    }
    if (!active) return;
    TransposeReduce<T, NV, 16>::run(acc, lane);
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) acc64[e] += (double)acc[e];
    double *dst = partial + ((int64_t)xr * P.ntiles + tile) * NV;
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) dst[lane * PER_LANE + e] = acc64[e];
}

template <int TM, int TN>
__global__ void gram_reduce_kernel(const double *partial, int nxr, int ntiles, int ct, int na, int nb,
                                   double *out) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= na * nb) return;
    const int i = o / nb, j = o % nb;
    const int tile = (i / TM) * ct + (j / TN);
    const int e = (i % TM) * TN + (j % TN);
    double s = 0.0;
    for (int x = 0; x < nxr; ++x) s += partial[((int64_t)x * ntiles + tile) * (TM * TN) + e];
    out[o] = s;
}

template <typename T>
static int run_gram(cnpc_ctx *ctx, int64_t ncell, const T *g, const T *fields, int64_t stride,
                    const int *a, int na, const int *b, int nb, double *out, cudaStream_t s) {
    constexpr int TM = TileShape<T>::TM, TN = TileShape<T>::TN;
    GramParams P;
    std::memset(&P, 0, sizeof(P));
    P.na = na;
    P.nb = nb;
    std::map<int, int> slot;
    for (int i = 0; i < na; ++i) {
        auto it = slot.find(a[i]);
        if (it == slot.end()) it = slot.emplace(a[i], (int)slot.size()).first;
        P.a_slot[i] = it->second + 1;  // slot 0 is G
    }
    for (int j = 0; j < nb; ++j) {
        auto it = slot.find(b[j]);
        if (it == slot.end()) it = slot.emplace(b[j], (int)slot.size()).first;
        P.b_slot[j] = it->second + 1;
    }
    CNPC_REQUIRE(ctx, (int)slot.size() <= kMaxUnion, "too many distinct fields (max 256)");
    P.nunion = (int)slot.size();
    for (auto &kv : slot) P.union_field[kv.second] = kv.first;
    const int rtiles = (na + TM - 1) / TM;
    P.ct = (nb + TN - 1) / TN;
    P.ntiles = rtiles * P.ct;
    P.ngroups = (P.ntiles + kWarps - 1) / kWarps;
    P.ncell = ncell;
    P.field_stride = stride;
    // chunk length: fit the staged rows in ~96 KB of shared memory
    const size_t budget = 96 * 1024;
    int chunk = (int)(budget / ((size_t)(P.nunion + 1) * sizeof(T)));
    chunk = std::min(1024, chunk) / 32 * 32;
    if (chunk < 32) chunk = 32;
    P.chunk = chunk;
    P.flush_chunks = std::max(1, 2048 / chunk);  // ~64 cells per lane per FP32 partial
    const size_t smem = (size_t)(P.nunion + 1) * chunk * sizeof(T);
    int st0;
    P.vec_ok = (stride % 4 == 0) && ((uintptr_t)g % 16 == 0) && ((uintptr_t)fields % 16 == 0);
    st0 = check_cuda(ctx, cudaFuncSetAttribute(gram_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem), "gram smem attribute");
    if (st0) return st0;
    int64_t nchunks = (ncell + chunk - 1) / chunk;
    int64_t per_sm = std::max<size_t>(1, (200 * 1024) / std::max<size_t>(smem, 1));
    per_sm = std::min<int64_t>(per_sm, 4);
    int64_t nxr = std::max<int64_t>(1, (int64_t)ctx->num_sms * per_sm / P.ngroups);
    nxr = std::min<int64_t>(nxr, nchunks);
    if (nxr < 1) nxr = 1;
    const size_t partial_bytes = (size_t)nxr * P.ntiles * TM * TN * sizeof(double);
    int st = ensure_scratch(ctx, partial_bytes, s);
    if (st) return st;
    gram_kernel<T><<<(unsigned)(nxr * P.ngroups), kThreads, smem, s>>>(g, fields, P, (double *)ctx->scratch);
    st = check_launch(ctx, "gram_kernel");
    if (st) return st;
    const int nout = na * nb;
    gram_reduce_kernel<TM, TN><<<(nout + 127) / 128, 128, 0, s>>>((const double *)ctx->scratch, (int)nxr,
                                                                  P.ntiles, P.ct, na, nb, out);
    return check_launch(ctx, "gram_reduce_kernel");
}

static int check_contract(cnpc_ctx *ctx, int dtype, int64_t ncell, const void *g, const void *f,
                          int64_t stride) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    CNPC_REQUIRE(ctx, ncell >= 1, "ncell must be >= 1");
    CNPC_REQUIRE(ctx, g && f, "null field pointer");
    CNPC_REQUIRE(ctx, stride >= ncell, "field_stride must be >= ncell");
    return CNPC_OK;
}

}  // namespace cnpc

using namespace cnpc;

extern "C" {

int cnpc_contract_gram(cnpc_ctx *ctx, int dtype, int64_t ncell, const void *d_g,
                       const void *d_fields, int64_t field_stride, const int *h_a, int na,
                       const int *h_b, int nb, double *d_out, cnpc_stream_t stream) {
    int st = check_contract(ctx, dtype, ncell, d_g, d_fields, field_stride);
    if (st) return st;
    CNPC_REQUIRE(ctx, h_a && h_b && d_out, "null argument");
    CNPC_REQUIRE(ctx, na >= 1 && na <= kMaxRows && nb >= 1 && nb <= kMaxRows, "na, nb must be 1..128");
    for (int i = 0; i < na; ++i) CNPC_REQUIRE(ctx, h_a[i] >= 0, "negative field index");
    for (int j = 0; j < nb; ++j) CNPC_REQUIRE(ctx, h_b[j] >= 0, "negative field index");
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == CNPC_F32)
        return run_gram<float>(ctx, ncell, (const float *)d_g, (const float *)d_fields, field_stride,
                               h_a, na, h_b, nb, d_out, s);
    return run_gram<double>(ctx, ncell, (const double *)d_g, (const double *)d_fields, field_stride,
                            h_a, na, h_b, nb, d_out, s);
}

}  // extern "C"
