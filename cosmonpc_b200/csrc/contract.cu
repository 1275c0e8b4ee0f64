// x-space triple-product reductions  sum_x G(x) F_a(x) F_b(x).
//
// Gram form: rows a_0..a_{na-1}, columns b_0..b_{nb-1}.  Each warp owns one
// TM x TN output tile; its 32 lanes stride over the cells of a chunk that the
// block stages in shared memory (G plus every field of the call).
//
// Staging: the chunk of each row is contiguous in HBM, so one elected thread
// copies it with cp.async.bulk (the TMA engine's linear copy) into a
// double-buffered shared-memory ring; an mbarrier with an expected byte count
// tells the 16 warps when a stage has landed.  The next chunk streams in while
// the current one is contracted.  Every mbarrier wait is bounded: a wait that
// gives up records CNPC_ETIMEOUT in the status word, the block drains its own
// copies (again bounded) and its outputs become NaN.
//
// Accumulation: FP32 fields accumulate TM*TN products per lane in FP32 for
// about 64 cells, then the warp folds the 32 lane partials with a
// recursive-halving shuffle transpose (lane l ends with tile elements 2l, 2l+1)
// and adds them into FP64 registers.  FP64 fields accumulate in FP64
// throughout.  Each block writes its FP64 tile partials; a second kernel sums
// them in a fixed order, so results are bitwise reproducible.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace cnpc {

constexpr int kWarps = 16;
constexpr int kThreads = kWarps * 32;
constexpr int kMaxRows = 128;
constexpr int kMaxUnion = 256;
constexpr long long kWaitLimit = 1ll << 22;  // try_wait polls before giving up (~seconds)

template <typename T> struct TileShape;
template <> struct TileShape<float> { static constexpr int TM = 8, TN = 8; };
template <> struct TileShape<double> { static constexpr int TM = 8, TN = 4; };

struct GramParams {
    int na, nb, nunion, ct, ntiles, ngroups, chunk, flush_chunks, async_ok;
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

// ------------------------------------------------------------ PTX helpers
__device__ inline uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ inline void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ inline void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ inline bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait; returns false if the barrier phase never completed.
__device__ inline bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ inline void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ inline void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <typename T>
__global__ void __launch_bounds__(kThreads) gram_kernel(const T *__restrict__ g,
                                                        const T *__restrict__ fields,
                                                        const GramParams P, double *partial,
                                                        int *status) {
    constexpr int TM = TileShape<T>::TM, TN = TileShape<T>::TN, NV = TM * TN;
    constexpr int PER_LANE = NV / 32;  // tile elements owned by a lane after the fold
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int abort_flag;
    const int nf = P.nunion + 1;  // staged rows: G then the union fields
    const int64_t stage_elems = (int64_t)nf * P.chunk;
    T *const stage0 = reinterpret_cast<T *>(smem_raw);

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
    for (int r = 0; r < TM; ++r) rs[r] = P.a_slot[min(rt * TM + r, P.na - 1)] * P.chunk;
#pragma unroll
    for (int c = 0; c < TN; ++c) cs[c] = P.b_slot[min(cti * TN + c, P.nb - 1)] * P.chunk;

    T acc[NV];
#pragma unroll
    for (int e = 0; e < NV; ++e) acc[e] = (T)0;
    double acc64[PER_LANE];
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) acc64[e] = 0.0;

    const int64_t first = (int64_t)xr * P.chunk;
    const int64_t step = (int64_t)nxr * P.chunk;
    const bool use_async = P.async_ok != 0;

    // issue the bulk copies of the chunk starting at c0 into stage s (one thread)
    auto issue = [&](int64_t c0, int s) {
        const int64_t valid = min((int64_t)P.chunk, P.ncell - c0);
        const uint32_t bytes = (uint32_t)(valid * sizeof(T));
        fence_proxy_async();
        mbar_expect_tx(&bars[s], bytes * (uint32_t)nf);
        for (int u = 0; u < nf; ++u) {
            const T *src = u == 0 ? g + c0 : fields + (int64_t)P.union_field[u - 1] * P.field_stride + c0;
            bulk_g2s(stage0 + s * stage_elems + (int64_t)u * P.chunk, src, bytes, &bars[s]);
        }
    };

    if (threadIdx.x == 0) {
        abort_flag = 0;
        if (use_async) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();
    if (use_async && threadIdx.x == 0 && first < P.ncell) issue(first, 0);

    int since_flush = 0;
    int it = 0;
    int64_t issued_last = first;  // start of the newest chunk whose copies were issued
    for (int64_t c0 = first; c0 < P.ncell; c0 += step, ++it) {
        const int s = it & 1;
        const int64_t valid = min((int64_t)P.chunk, P.ncell - c0);
        T *sb = stage0 + s * stage_elems;
        if (use_async) {
            // prefetch the next chunk into the other stage (freed by the
            // __syncthreads at the end of the previous iteration)
            if (threadIdx.x == 0 && c0 + step < P.ncell && !abort_flag) {
                issue(c0 + step, s ^ 1);
                issued_last = c0 + step;
            }
            if (threadIdx.x == 0) {
                if (!mbar_wait_bounded(&bars[s], (uint32_t)((it >> 1) & 1))) {
                    abort_flag = 1;
                    atomicExch(status, (int)CNPC_ETIMEOUT);
                }
            }
            __syncthreads();
            if (abort_flag) break;
            // the other threads observe the completed phase through the barrier
            // wait of thread 0 plus __syncthreads; re-check the phase locally to
            // get acquire semantics on the copied bytes
            mbar_try_wait(&bars[s], (uint32_t)((it >> 1) & 1));
        } else {
            __syncthreads();
            for (int idx = threadIdx.x; idx < nf * P.chunk; idx += kThreads) {
                const int u = idx / P.chunk, c = idx % P.chunk;
                const int64_t cell = c0 + c;
                T v = (T)0;
                if (cell < P.ncell)
                    v = u == 0 ? g[cell] : fields[(int64_t)P.union_field[u - 1] * P.field_stride + cell];
                sb[(int64_t)u * P.chunk + c] = v;
            }
            __syncthreads();
        }
        if (active) {
            for (int c = lane; c < valid; c += 32) {
                const T gv = sb[c];
                T av[TM], bv[TN];
#pragma unroll
                for (int r = 0; r < TM; ++r) av[r] = gv * sb[rs[r] + c];
#pragma unroll
                for (int q = 0; q < TN; ++q) bv[q] = sb[cs[q] + c];
#pragma unroll
                for (int r = 0; r < TM; ++r)
#pragma unroll
                    for (int q = 0; q < TN; ++q) acc[r * TN + q] += av[r] * bv[q];
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
        __syncthreads();  // every warp is done with stage s before it is refilled
    }
    if (use_async && abort_flag && threadIdx.x == 0) {
        // drain the copies this block still has in flight (bounded) before
        // exit: the chunk whose wait gave up and the newest prefetched chunk
        mbar_wait_bounded(&bars[it & 1], (uint32_t)((it >> 1) & 1));
        const int itl = (int)((issued_last - first) / step);
        if (itl != it) mbar_wait_bounded(&bars[itl & 1], (uint32_t)((itl >> 1) & 1));
    }
    __syncthreads();
    if (!active) return;
    TransposeReduce<T, NV, 16>::run(acc, lane);
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) acc64[e] += (double)acc[e];
    double *dst = partial + ((int64_t)xr * P.ntiles + tile) * NV;
    const double nanv = __longlong_as_double(0x7ff8000000000000ll);
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) dst[lane * PER_LANE + e] = abort_flag ? nanv : acc64[e];
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
    // bulk copies need 16-byte aligned sources and byte counts
    P.async_ok = ((stride * sizeof(T)) % 16 == 0) && ((ncell * sizeof(T)) % 16 == 0) &&
                 ((uintptr_t)g % 16 == 0) && ((uintptr_t)fields % 16 == 0);
    // two stages of (G + union rows) x chunk in ~100 KB of shared memory
    const size_t budget = 100 * 1024;
    int chunk = (int)(budget / (2 * (size_t)(P.nunion + 1) * sizeof(T)));
    chunk = std::min(1024, chunk) / 32 * 32;
    if (chunk < 32) chunk = 32;
    P.chunk = chunk;
    P.flush_chunks = std::max(1, 2048 / chunk);  // ~64 cells per lane per FP32 partial
    const size_t smem = 2 * (size_t)(P.nunion + 1) * chunk * sizeof(T);
    int st = check_cuda(ctx, cudaFuncSetAttribute(gram_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem), "gram smem attribute");
    if (st) return st;
    const int64_t nchunks = (ncell + chunk - 1) / chunk;
    int per_sm = (int)std::max<size_t>(1, (220 * 1024) / std::max<size_t>(smem + 1024, 1));
    per_sm = std::min(per_sm, 2);
    int64_t nxr = std::max<int64_t>(1, (int64_t)ctx->num_sms * per_sm / P.ngroups);
    nxr = std::min<int64_t>(nxr, nchunks);
    const size_t partial_bytes = (size_t)nxr * P.ntiles * TM * TN * sizeof(double) + 256;
    st = ensure_scratch(ctx, partial_bytes, s);
    if (st) return st;
    int *status = reinterpret_cast<int *>(static_cast<char *>(ctx->scratch) + ctx->scratch_bytes - 256);
    gram_kernel<T><<<(unsigned)(nxr * P.ngroups), kThreads, smem, s>>>(g, fields, P, (double *)ctx->scratch,
                                                                        status);
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
