// FP32 Gram contraction on the 5th-generation tensor cores (tcgen05, TF32 pairs).
//
//   out[i][j] = sum_x G(x) F_{a_i}(x) F_{b_j}(x),  i < na <= 64, j < nb <= 32
//
// is a GEMM D = A B^T with rows A_i = G F_{a_i}, columns B_j = F_{b_j} and
// K = cells, K-major on both sides because every field row is contiguous over
// cells.  Each FP32 operand is split into a TF32 pair x = hi + lo
// (Veltkamp split with 2^13 + 1: hi keeps 11 significant bits, lo = x - hi
// exactly, |lo| <= 2^-12 |x|; the tensor core's TF32 view of lo drops at most
// 2^-23 |x|), and ONE MMA per K-step of 8 cells takes all four
// products: A' = [A_hi ; A_lo] (M = 128 rows), B' = [B_hi ; B_lo] (N = 2n), so
//   D[i][j] + D[i][n+j] + D[64+i][j] + D[64+i][n+j] = (A_hi+A_lo)(B_hi+B_lo).
//
// Per CTA (one per SM, persistent over chunks of 64 cells): 16 warps load the
// chunk's rows (8 fields x 16 cells per warp item, registers double-buffered
// one chunk ahead), multiply A rows by G, split (Veltkamp, FP32 arithmetic
// only), and store hi/lo into the K-major 128-byte-swizzled UMMA layout (atoms
// of 8 rows x 32 cells, 16-byte chunk c of row r at c ^ r, 1024 B between row
// groups; the 8 lanes of one quad store to 8 distinct bank groups) of one
// of two shared-memory buffers; one thread issues the chunk's 8 MMAs and
// commits them to the buffer's mbarrier, which the loaders wait on before
// refilling the buffer two chunks later.  Consecutive K-steps go to 4
// independent TMEM accumulators (so the tensor pipe never waits on its own
// previous result), and the accumulator set alternates every 4 chunks: a
// finished set is read with tcgen05.ld and added into FP64 registers, so FP32
// only ever sums 64 cells of one accumulator.  Per-CTA FP64 partials are
// reduced in a fixed order.
//
// Every mbarrier wait is bounded; a wait that gives up makes the CTA's
// partials NaN, stops issuing MMAs, drains (again bounded) and frees its TMEM.
#include <algorithm>
#include <cstring>

#include "internal.h"

namespace cnpc {
namespace tc {

constexpr int kThreads = 512;        // 16 warps
constexpr int kChunk = 64;           // cells per chunk (8 K-steps)
constexpr int kKSteps = kChunk / 8;
constexpr int kPeriod = 4;           // chunks per accumulator set
constexpr int kChains = 4;           // independent accumulators per set
constexpr int kMaxRowsTc = 64;
constexpr int kMaxColsTc = 32;
constexpr int kAtom = 16 * 1024;     // A' K-atom (32 cells): 16 row groups (hi 0-7, lo 8-15) x 1024 B
constexpr int kAPlane = 2 * kAtom;   // the chunk's two K-atoms
constexpr long long kSpinLimit = 1ll << 22;

struct TcParams {
    int na, nb, n, na8, nb8, ngroups, tmem_cols;
    int64_t ncell, stride;
    int a_slot[kMaxRowsTc];
    int b_slot[kMaxColsTc];
};

__device__ inline uint32_t saddr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ inline uint64_t umma_desc(uint32_t addr) {
    // K-major, 128-byte swizzle: start >> 4 | LBO 16 B (unused) | SBO 1024 B >> 4 << 32 |
    // version 1 (bit 46) | layout SWIZZLE_128B = 2 (bits 61-63); atoms 1024-byte aligned
    return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
    // D F32 (bits 4-5), A and B TF32 (bits 7-9, 10-12), both K-major, N >> 3 at 17, M >> 4 at 24
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ inline void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ inline void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ inline void bar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}

__device__ inline bool bar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ inline bool bar_wait(uint64_t *bar, uint32_t parity) {
    for (long long i = 0; i < kSpinLimit; ++i)
        if (bar_try(bar, parity)) return true;
    return false;
}

// Veltkamp split (Dekker 1971): p = x (2^13 + 1), hi = p - (p - x) keeps the
// 11 leading bits of x rounded to nearest, lo = x - hi exactly
__device__ inline void split1(float x, uint32_t &hi, uint32_t &lo) {
    const float p = __fmul_rn(x, 8193.0f);
    const float h = __fsub_rn(p, __fsub_rn(p, x));
    hi = __float_as_uint(h);
    lo = __float_as_uint(__fsub_rn(x, h));
}
__device__ inline void split4(float4 x, uint4 &hi, uint4 &lo) {
    split1(x.x, hi.x, lo.x), split1(x.y, hi.y, lo.y), split1(x.z, hi.z, lo.z), split1(x.w, hi.w, lo.w);
}

__device__ inline void tmem_ld4(uint32_t taddr, float *v) {
    uint32_t r0, r1, r2, r3;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(taddr));
    v[0] = __uint_as_float(r0), v[1] = __uint_as_float(r1), v[2] = __uint_as_float(r2), v[3] = __uint_as_float(r3);
}
__device__ inline void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

constexpr int kItems = 3;  // warp items per chunk per warp: 12 groups x 4 cell blocks / 16 warps

__global__ void __launch_bounds__(kThreads, 1)
    gram_tc_kernel(const float *__restrict__ g, const float *__restrict__ fields, const TcParams P,
                   double *__restrict__ partial) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // swizzle atoms need 1024-byte aligned shared addresses
    unsigned char *smem = smem_raw + ((1024 - (saddr(smem_raw) & 1023)) & 1023);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n2 = 2 * P.n;
    const int batom = 2 * P.nb8 * 1024;                // B' K-atom: 2n rows (hi, then lo) x 128 B
    const int buf_bytes = kAPlane + 2 * batom;           // A' and B' of one chunk
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * buf_bytes);
    uint32_t *taddr_slot = reinterpret_cast<uint32_t *>(bars + 2);

    // zero both buffers once (padding rows feed only discarded outputs, but stay finite)
    for (int i = tid; i < 2 * buf_bytes / 16; i += kThreads)
        reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        bar_init(&bars[0]);
        bar_init(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(taddr_slot)),
                     "r"(P.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *taddr_slot;

    const int64_t nchunk_all = (P.ncell + kChunk - 1) / kChunk;
    const int nchunk = blockIdx.x < nchunk_all ? (int)((nchunk_all - 1 - blockIdx.x) / gridDim.x + 1) : 0;

    // warp item geometry: cell block cb (16 cells), groups gset + 4k; lane = field in
    // group (lane & 7) x quad in block (lane >> 3)
    const int cb = warp & 3, gset = warp >> 2;
    const int f8 = lane & 7, qd = lane >> 3;
    const int katom = cb >> 1, kchunk = (cb & 1) * 4 + qd;  // K-atom and 16-byte chunk of the lane's quad
    const int in_group = f8 * 128 + ((kchunk ^ f8) << 4);  // swizzled offset inside a row group

    // fold geometry: quadrant q = warp & 3 reads TMEM lanes 32q..32q+31 (D rows: lane L
    // is A' row L), column slice h = warp >> 2 of each accumulator's 2n columns
    const int q = warp & 3, h = warp >> 2;
    const int wcols = n2 / 4;  // multiple of 4 (n is a multiple of 8)
    double acc64[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc64[c] = 0.0;
    bool ok = true;

    auto load_chunk = [&](int i, float4 *v, float4 &gq) {
        const int64_t chunk = (int64_t)blockIdx.x + (int64_t)i * gridDim.x;
        const int64_t cell = chunk * kChunk + (cb * 4 + qd) * 4;
        const bool in = cell < P.ncell;  // ncell is a multiple of 4
        gq = in ? __ldg(reinterpret_cast<const float4 *>(g + cell)) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const int gi = gset + 4 * k;
            int field = -1;
            if (gi < P.na8) {
                const int r = gi * 8 + f8;
                if (r < P.na) field = P.a_slot[r];
            } else if (gi < P.ngroups) {
                const int c = (gi - P.na8) * 8 + f8;
                if (c < P.nb) field = P.b_slot[c];
            }
            v[k] = (in && field >= 0) ? __ldg(reinterpret_cast<const float4 *>(fields + (int64_t)field * P.stride + cell))
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };

    auto store_chunk = [&](unsigned char *b, const float4 *v, float4 gq) {
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const int gi = gset + 4 * k;
            if (gi >= P.ngroups) continue;
            uint4 hi, lo;
            if (gi < P.na8) {
                const float4 x = make_float4(v[k].x * gq.x, v[k].y * gq.y, v[k].z * gq.z, v[k].w * gq.w);
                split4(x, hi, lo);
                const int off = katom * kAtom + gi * 1024 + in_group;
                *reinterpret_cast<uint4 *>(b + off) = hi;
                *reinterpret_cast<uint4 *>(b + off + 8 * 1024) = lo;
            } else {
                split4(v[k], hi, lo);
                const int gb = gi - P.na8;
                const int off = kAPlane + katom * batom + gb * 1024 + in_group;
                *reinterpret_cast<uint4 *>(b + off) = hi;
                *reinterpret_cast<uint4 *>(b + off + P.nb8 * 1024) = lo;
            }
        }
    };

    auto fold = [&](int period) {
        tc_fence_after();
        const uint32_t set = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)((period & 1) * kChains * n2 + h * wcols);
#pragma unroll 1
        for (int c = 0; c < kChains; ++c) {
            float v[16];
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4)
                if (c4 * 4 < wcols) tmem_ld4(set + c * n2 + c4 * 4, v + c4 * 4);
            tmem_wait_ld();
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (k < wcols) acc64[k] += (double)v[k];
        }
    };

    const uint32_t idesc = idesc_tf32(128, n2);
    float4 cur[kItems], nxt[kItems], gcur, gnxt;
    if (nchunk > 0) load_chunk(0, cur, gcur);
    for (int i = 0; i < nchunk; ++i) {
        const int b = i & 1;
        if (i + 1 < nchunk) load_chunk(i + 1, nxt, gnxt);
        if (i >= 2) {
            // the MMAs of chunk i - 2 read this buffer; their period may be finished
            const int j = i - 2;
            if (ok && !bar_wait(&bars[b], (uint32_t)((j >> 1) & 1))) ok = false;
            ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld below is warp-collective
            if (ok && (j % kPeriod == kPeriod - 1)) fold(j / kPeriod);
        }
        if (ok) store_chunk(smem + b * buf_bytes, cur, gcur);
        proxy_fence();
        tc_fence_before();
        ok = __syncthreads_and(ok);
        if (ok && tid == 0) {
            tc_fence_after();
            const uint32_t a0 = saddr(smem + b * buf_bytes);
            const uint32_t dset = tmem + (uint32_t)(((i / kPeriod) & 1) * kChains * n2);
            const bool first = (i % kPeriod) == 0;
#pragma unroll
            for (int ks = 0; ks < kKSteps; ++ks) {
                const uint32_t kin = (ks & 3) * 32;  // K-step inside the swizzle atom
                const uint64_t ad = umma_desc(a0 + (ks >> 2) * kAtom + kin);
                const uint64_t bd = umma_desc(a0 + kAPlane + (ks >> 2) * batom + kin);
                mma_tf32(dset + (ks % kChains) * n2, ad, bd, idesc, (first && ks < kChains) ? 0u : 1u);
            }
            mma_commit(&bars[b]);
        }
#pragma unroll
        for (int k = 0; k < kItems; ++k) cur[k] = nxt[k];
        gcur = gnxt;
    }
    // drain: the last two chunks' MMAs, then their periods
    for (int j = nchunk - 2 > 0 ? nchunk - 2 : 0; j < nchunk; ++j) {
        // waited even after a failure, so that no MMA is in flight when TMEM is freed
        if (!bar_wait(&bars[j & 1], (uint32_t)((j >> 1) & 1))) ok = false;
        ok = __all_sync(0xffffffffu, ok);
        if (ok && (j % kPeriod == kPeriod - 1 || j == nchunk - 1)) fold(j / kPeriod);
    }
    // a period that ended on chunk nchunk - 3 or earlier was folded in the loop;
    // one that ends on the last chunk was folded just now
    ok = __syncthreads_and(ok);
    {
        const int L = 32 * q + lane;  // A' row: hi row L for L < 64, lo row L - 64 after
        double *dst = partial + ((int64_t)blockIdx.x * 128 + L) * (2 * kMaxColsTc) + h * wcols;
        const double nanv = __longlong_as_double(0x7ff8000000000000ll);
#pragma unroll
        for (int c = 0; c < 16; ++c)
            if (c < wcols) dst[c] = ok ? acc64[c] : nanv;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P.tmem_cols));
    }
}

// out[i * nb + j] = sum over blocks of the four TF32 products hi.hi, hi.lo,
// lo.hi, lo.lo of (i, j), one warp per output, fixed order
__global__ void gram_tc_reduce_kernel(const double *partial, int nblocks, int na, int nb, int n, double *out) {
    const int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= na * nb) return;
    const int i = o / nb, j = o % nb;
    double s = 0.0;
    for (int p = lane; p < nblocks; p += 32) {
        const double *hi = partial + ((int64_t)p * 128 + i) * (2 * kMaxColsTc);
        const double *lo = hi + 64 * (2 * kMaxColsTc);
        s += (hi[j] + hi[n + j]) + (lo[j] + lo[n + j]);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) out[o] = s;
}

}  // namespace tc
}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_contract_gram_tc(cnpc_ctx *ctx, int64_t ncell, const float *d_g, const float *d_fields,
                                     int64_t field_stride, const int *h_a, int na, const int *h_b, int nb,
                                     double *d_out, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, d_g && d_fields && d_out && h_a && h_b, "null argument");
    CNPC_REQUIRE(ctx, na >= 1 && na <= tc::kMaxRowsTc && nb >= 1 && nb <= tc::kMaxColsTc,
                 "tensor-core Gram covers 1..64 rows x 1..32 columns");
    CNPC_REQUIRE(ctx, ncell > 0 && ncell % 4 == 0 && field_stride >= ncell && field_stride % 4 == 0,
                 "ncell and field_stride must be positive multiples of 4, field_stride >= ncell");
    CNPC_REQUIRE(ctx, (uintptr_t)d_g % 16 == 0 && (uintptr_t)d_fields % 16 == 0, "G and fields must be 16-byte aligned");
    tc::TcParams P;
    std::memset(&P, 0, sizeof(P));
    P.na = na;
    P.nb = nb;
    P.n = (nb + 7) / 8 * 8;
    P.na8 = (na + 7) / 8;
    P.nb8 = P.n / 8;
    P.ngroups = P.na8 + P.nb8;
    P.ncell = ncell;
    P.stride = field_stride;
    for (int i = 0; i < na; ++i) {
        CNPC_REQUIRE(ctx, h_a[i] >= 0, "negative field index");
        P.a_slot[i] = h_a[i];
    }
    for (int j = 0; j < nb; ++j) {
        CNPC_REQUIRE(ctx, h_b[j] >= 0, "negative field index");
        P.b_slot[j] = h_b[j];
    }
    int cols = 32;
    while (cols < 2 * tc::kChains * 2 * P.n) cols *= 2;
    P.tmem_cols = cols;
    const size_t buf_bytes = (size_t)tc::kAPlane + 2 * (size_t)(2 * P.nb8 * 1024);
    const size_t smem = 2 * buf_bytes + 64 + 1024;
    const int64_t nchunks = (ncell + tc::kChunk - 1) / tc::kChunk;
    const int nblocks = (int)std::min<int64_t>(ctx->num_sms, nchunks);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t part_bytes = (size_t)nblocks * 128 * 2 * tc::kMaxColsTc * sizeof(double);
    int st = ensure_scratch(ctx, part_bytes, s);
    if (st) return st;
    double *part = (double *)ctx->scratch;
    st = check_cuda(ctx, cudaFuncSetAttribute(tc::gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "gram_tc_kernel smem");
    if (st) return st;
    tc::gram_tc_kernel<<<nblocks, tc::kThreads, smem, s>>>(d_g, d_fields, P, part);
    st = check_launch(ctx, "gram_tc_kernel");
    if (st) return st;
    const int nout = na * nb;
    tc::gram_tc_reduce_kernel<<<(nout + 7) / 8, 256, 0, s>>>(part, nblocks, na, nb, P.n, d_out);
    return check_launch(ctx, "gram_tc_reduce_kernel");
}
