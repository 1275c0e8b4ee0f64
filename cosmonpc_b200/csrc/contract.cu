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
    int na, nb, nunion, ct, ntiles, ngroups, chunk, flush_chunks;
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

__device__ inline void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

constexpr int kStages = 4;

// Tiles handled by block group g and the warp -> (tile, phase) map: the tiles
// of a group are spread over the 16 warps; a tile with several warps splits
// its cells between them (phase p of n takes every n-th 32-cell slice).
struct WarpWork {
    int tile, phase, nphase;
};
__device__ inline WarpWork warp_work(int group, int warp, int ntiles) {
    const int t0 = group * kWarps;
    const int nt = min(kWarps, ntiles - t0);
    WarpWork w;
    w.tile = t0 + warp % nt;
    w.phase = warp / nt;
    w.nphase = (kWarps - 1 - warp % nt) / nt + 1;
    return w;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) gram_kernel(const T *__restrict__ g,
                                                        const T *__restrict__ fields,
                                                        const GramParams P, double *partial,
                                                        int *status) {
    constexpr int TM = TileShape<T>::TM, TN = TileShape<T>::TN, NV = TM * TN;
    constexpr int PER_LANE = NV / 32;  // tile elements owned by a lane after the fold
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kStages];
    __shared__ __align__(8) uint64_t empty_bar[kStages];
    __shared__ volatile int abort_flag;
    const int nf = P.nunion + 1;  // staged rows: G then the union fields
    const int64_t stage_elems = (int64_t)nf * P.chunk;
    T *const stage0 = reinterpret_cast<T *>(smem_raw);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int group = blockIdx.x % P.ngroups;
    const int xr = blockIdx.x / P.ngroups;
    const int nxr = gridDim.x / P.ngroups;
    const WarpWork ww = warp_work(group, warp, P.ntiles);
    const int rt = ww.tile / P.ct;
    const int cti = ww.tile % P.ct;

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
    const int nchunk = first < P.ncell ? (int)((P.ncell - first + step - 1) / step) : 0;
    const bool producer = threadIdx.x == 0;

    auto issue = [&](int k) {  // bulk copies of this block's k-th chunk
        const int s = k % kStages;
        const int64_t c0 = first + (int64_t)k * step;
        const int64_t valid = min((int64_t)P.chunk, P.ncell - c0);
        const uint32_t bytes = (uint32_t)(valid * sizeof(T));
        T *dst = stage0 + s * stage_elems;
        fence_proxy_async();
        mbar_expect_tx(&full_bar[s], bytes * (uint32_t)nf);
        for (int u = 0; u < nf; ++u) {
            const T *src = u == 0 ? g + c0 : fields + (int64_t)P.union_field[u - 1] * P.field_stride + c0;
            bulk_g2s(dst + (int64_t)u * P.chunk, src, bytes, &full_bar[s]);
        }
    };

    if (producer) {
        abort_flag = 0;
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = 0;
    if (producer)
        for (; issued < min(nchunk, kStages - 1); ++issued) issue(issued);

    int since_flush = 0;
    int k = 0;
    for (; k < nchunk; ++k) {
        const int s = k % kStages;
        // producer: refill the stage freed by chunk k-1 with chunk k+kStages-1
        if (producer && issued < nchunk && !abort_flag) {
            const int sp = issued % kStages;
            if (issued >= kStages && !mbar_wait_bounded(&empty_bar[sp], (uint32_t)(((issued / kStages) - 1) & 1))) {
                abort_flag = 1;
                atomicExch(status, (int)CNPC_ETIMEOUT);
            } else {
                issue(issued);
                ++issued;
            }
        }
        if (!mbar_wait_bounded(&full_bar[s], (uint32_t)((k / kStages) & 1))) {
            abort_flag = 1;
            if (lane == 0) atomicExch(status, (int)CNPC_ETIMEOUT);
        }
        if (abort_flag) break;
        const T *sb = stage0 + s * stage_elems;
        const int64_t valid = min((int64_t)P.chunk, P.ncell - (first + (int64_t)k * step));
        const int cstep = 32 * ww.nphase;
        for (int c = lane + 32 * ww.phase; c < (int)valid; c += cstep) {
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
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[s]);
        if (sizeof(T) == 4 && ++since_flush == P.flush_chunks) {
            since_flush = 0;
            TransposeReduce<T, NV, 16>::run(acc, lane);
#pragma unroll
            for (int e = 0; e < PER_LANE; ++e) acc64[e] += (double)acc[e];
#pragma unroll
            for (int e = 0; e < NV; ++e) acc[e] = (T)0;
        }
    }
    if (abort_flag && producer) {
        // drain the copies still in flight (bounded) before the block exits
        for (int j = k; j < issued; ++j) mbar_wait_bounded(&full_bar[j % kStages], (uint32_t)((j / kStages) & 1));
    }
    TransposeReduce<T, NV, 16>::run(acc, lane);
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) acc64[e] += (double)acc[e];
    // per-warp partials: [block][warp][NV]
    double *dst = partial + ((int64_t)blockIdx.x * kWarps + warp) * NV;
    const double nanv = __longlong_as_double(0x7ff8000000000000ll);
    const bool bad = abort_flag != 0;
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) dst[lane * PER_LANE + e] = bad ? nanv : acc64[e];
}

// out[i, j] = sum over every block of the group owning tile(i, j) and every
// warp of that block assigned to the tile, in a fixed order.
template <int TM, int TN>
__global__ void gram_reduce_kernel(const double *partial, int nblocks, int ngroups, int ntiles, int ct,
                                   int na, int nb, double *out) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= na * nb) return;
    const int i = o / nb, j = o % nb;
    const int tile = (i / TM) * ct + (j / TN);
    const int e = (i % TM) * TN + (j % TN);
    const int group = tile / kWarps;
    const int nt = min(kWarps, ntiles - group * kWarps);
    const int local = tile - group * kWarps;
    double s = 0.0;
    for (int b = group; b < nblocks; b += ngroups)
        for (int w = local; w < kWarps; w += nt) s += partial[((int64_t)b * kWarps + w) * (TM * TN) + e];
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
    CNPC_REQUIRE(ctx, ((stride * sizeof(T)) % 16 == 0) && ((ncell * sizeof(T)) % 16 == 0) &&
                          ((uintptr_t)g % 16 == 0) && ((uintptr_t)fields % 16 == 0),
                 "contraction needs 16-byte aligned fields, field_stride and ncell");
    // kStages x (G + union rows) x chunk in ~200 KB of shared memory (1 block/SM)
    const size_t budget = 200 * 1024;
    int chunk = (int)(budget / (kStages * (size_t)(P.nunion + 1) * sizeof(T)));
    chunk = std::min(1024, chunk) / 32 * 32;
    CNPC_REQUIRE(ctx, chunk >= 32, "too many distinct fields for the shared-memory stages");
    P.chunk = chunk;
    P.flush_chunks = std::max(1, 2048 / chunk);  // ~64 cells per lane per FP32 partial
    const size_t smem = (size_t)kStages * (P.nunion + 1) * chunk * sizeof(T);
    int st = check_cuda(ctx, cudaFuncSetAttribute(gram_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem), "gram smem attribute");
    if (st) return st;
    const int64_t nchunks = (ncell + chunk - 1) / chunk;
    int64_t nxr = std::min<int64_t>(std::max<int64_t>(1, ctx->num_sms / P.ngroups), nchunks);
    const int nblocks = (int)(nxr * P.ngroups);
    const size_t partial_bytes = (size_t)nblocks * kWarps * TM * TN * sizeof(double) + 256;
    st = ensure_scratch(ctx, partial_bytes, s);
    if (st) return st;
    int *status = reinterpret_cast<int *>(static_cast<char *>(ctx->scratch) + ctx->scratch_bytes - 256);
    gram_kernel<T><<<(unsigned)nblocks, kThreads, smem, s>>>(g, fields, P, (double *)ctx->scratch, status);
    st = check_launch(ctx, "gram_kernel");
    if (st) return st;
    const int nout = na * nb;
    gram_reduce_kernel<TM, TN><<<(nout + 127) / 128, 128, 0, s>>>((const double *)ctx->scratch, nblocks,
                                                                  P.ngroups, P.ntiles, P.ct, na, nb, out);
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
