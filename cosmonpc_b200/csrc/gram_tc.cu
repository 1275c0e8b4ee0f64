// FP32 Gram contraction on the 5th-generation tensor cores (tcgen05, TF32 pairs).
//
//   out[i][j] = sum_x G_{g_i}(x) F_{a_i}(x) F_{b_j}(x),  i < na <= 40, j < nb <= 24
//
// is a GEMM D = A B^T with rows A_i = G_{g_i} F_{a_i}, columns B_j = F_{b_j} and
// K = cells.  Each FP32 operand is split into a TF32 pair x = hi + lo
// (Veltkamp split with 2^13 + 1: hi keeps 11 significant bits, lo = x - hi
// exactly, |lo| <= 2^-12 |x|; the tensor core's TF32 view of lo drops at most
// 2^-23 |x|), and ONE MMA per K-step of 8 cells takes all four products:
// A' = [A_hi ; A_lo] (M = 128: rows 0..39 hi, 64..103 lo), B' = [B_hi ; B_lo]
// (N = 48: rows 0..23 hi, 24..47 lo), so
//   C[i][j] = D[i][j] + D[i][24+j] + D[64+i][j] + D[64+i][24+j].
//
// A' lives in tensor memory (the MMA's A-from-TMEM form), written by the
// converter warps with tcgen05.st straight from registers: the tensor core
// then reads only B' (48 x 4 bytes per cell) from shared memory, and no
// shared-memory pass carries the 40 A rows.  Warp roles (one CTA per SM,
// persistent over 32-cell chunks, chunk t of a CTA = cells
// 32 (blockIdx.x + t gridDim.x) ..):
//   * converter groups (kGroups x 4 warps; group t % kGroups takes chunk t):
//     TMEM lane L = 32 (warp % 4) + lane owns A' row L: it loads its field
//     row (and reads the chunk's weight field from a shared ring), forms
//     G F, splits, and stores its 32 values into the chunk's TMEM stage;
//     lanes with no A row (40..63, 104..127) split a B row into the chunk's
//     128-byte-swizzled K-major shared-memory stage.  Field rows are loaded
//     one chunk ahead into registers (no shared-memory staging).
//   * one MMA warp: its lane 0 copies the weight-field chunks into the ring
//     (cp.async.bulk, kStages ahead), waits for a stage's converters, issues
//     the 4 MMAs of the chunk and commits them to the stage's "empty"
//     mbarrier; the accumulator set alternates every kPeriod chunks and its
//     completion is committed to the fold warps.
//   * four fold warps read a finished accumulator set (tcgen05.ld), add
//     D[L][j] + D[L][24+j] into FP64 registers and release the set, so FP32
//     only ever sums one period (512 cells) of one accumulator.
// Per-CTA FP64 partials are reduced in a fixed order (bitwise reproducible).
//
// Every mbarrier wait is bounded (the context's wait limit): a wait that gives
// up sets the abort flag and the context's status word (CNPC_ETIMEOUT), every
// role stops, the MMA thread drains its own MMAs and copies (bounded by a
// fixed limit) before TMEM is freed, and the CTA's partials are NaN.
#include <algorithm>
#include <cstring>

#include "internal.h"

namespace cnpc {
namespace tc {

constexpr int kGroups = 2;                 // converter warp groups
constexpr int kStages = 8;                 // chunk stages in flight (TMEM A' + shared B'), a multiple of kGroups
constexpr int kThreads = 32 * (4 * kGroups + 4 + 1);
constexpr int kConvWarps = 4 * kGroups;
constexpr int kFoldWarp0 = kConvWarps;     // warps kFoldWarp0 .. +3 fold
constexpr int kMmaWarp = kConvWarps + 4;
constexpr int kChunk = 32;                 // cells per chunk: one 128-byte swizzle atom of K
constexpr int kPeriod = 16;                // chunks per accumulator set
constexpr int kMaxRowsTc = 40;
constexpr int kMaxColsTc = 24;
constexpr int kN = 48;                     // B' rows: hi 0..23, lo 24..47
constexpr int kBStage = kN / 8 * 1024;     // 6 row groups of 8 rows x 128 bytes
constexpr int kMaxGs = 4;
constexpr int kDCol = 64;                  // accumulator set p at TMEM column 64 p
constexpr int kACol0 = 128;                // A' stage s at TMEM column 128 + 32 s
constexpr int kTmemCols = (kACol0 + kStages * kChunk) <= 256 ? 256 : 512;
constexpr long long kDrainLimit = 1ll << 22;
constexpr int kPrefetch = 12;              // chunks of L2 prefetch ahead of the register loads
constexpr int kGRing = 16;                 // weight-field ring: copies issued kGRing chunks ahead

struct TcParams {
    int na, nb, ngs;
    int64_t ncell, stride;
    long long wait_limit;
    const float *g[kMaxGs];
    int a_slot[kMaxRowsTc];
    int a_g[kMaxRowsTc];
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

// D (TMEM) += A (TMEM) * B (shared memory)^T
__device__ inline void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                   uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ inline void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ inline void bar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ inline void bar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}
__device__ inline void bar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
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
// Bounded wait: false after `limit` polls, or as soon as another role aborted.
__device__ inline bool bar_wait(uint64_t *bar, uint32_t parity, long long limit, volatile int *abort_flag) {
    for (long long i = 0; i < limit; ++i) {
        if (bar_try(bar, parity)) return true;
        if (abort_flag && (i & 63) == 63 && *abort_flag) return false;
    }
    return false;
}
__device__ inline void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar))
        : "memory");
}

// Veltkamp split (Dekker 1971): p = x (2^13 + 1), hi = p - (p - x) keeps the
// 11 leading bits of x rounded to nearest, lo = x - hi exactly
__device__ inline float split_hi(float x) {
    const float p = __fmul_rn(x, 8193.0f);
    return __fsub_rn(p, __fsub_rn(p, x));
}

// 32 consecutive TMEM columns of this thread's lane
__device__ inline void tmem_st32(uint32_t taddr, const uint32_t *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(
            taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
        "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
        "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
        : "memory");
}
// 16 consecutive TMEM columns of this thread's lane
__device__ inline void tmem_st16(uint32_t taddr, const uint32_t *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ inline void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ inline void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ inline void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

struct __align__(8) TcShared {
    uint64_t full[kStages];    // converters of the chunk done (kConvWarpsPerGroup arrivals)
    uint64_t empty[kStages];   // the chunk's MMAs done (tcgen05.commit)
    uint64_t gfull[kGRing];    // a chunk's weight-field copies landed (tx count)
    uint64_t dfull[2];         // accumulator set complete (tcgen05.commit)
    uint64_t dempty[2];        // accumulator set folded (4 fold warps)
    uint64_t drain;
    uint32_t tmem_base;
    int abort_flag;
};

__global__ void __launch_bounds__(kThreads, 1)
    gram_tc_kernel(const float *__restrict__ fields, const TcParams P, double *__restrict__ partial, int *status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned B' stages, then the weight-field ring, then the barriers
    unsigned char *base = smem_raw + ((1024 - (saddr(smem_raw) & 1023)) & 1023);
    unsigned char *bstage = base;                                                  // [kStages][kBStage]
    float *gring = reinterpret_cast<float *>(base + kStages * kBStage);           // [kGRing][kMaxGs][kChunk]
    TcShared &S = *reinterpret_cast<TcShared *>(gring + kGRing * kMaxGs * kChunk);
    volatile int *abort_flag = &S.abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // each CTA takes a contiguous run of chunks, so that the rows it streams
    // can be prefetched into L2 a fixed distance ahead
    const int64_t nchunk_all = (P.ncell + kChunk - 1) / kChunk;
    const int64_t per_cta = (nchunk_all + gridDim.x - 1) / gridDim.x;
    const int64_t first_chunk = (int64_t)blockIdx.x * per_cta;
    const int nchunk = first_chunk < nchunk_all ? (int)min(per_cta, nchunk_all - first_chunk) : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            bar_init(&S.full[s], 4);
            bar_init(&S.empty[s], 1);
        }
        for (int r = 0; r < kGRing; ++r) bar_init(&S.gfull[r], 1);
        for (int p = 0; p < 2; ++p) {
            bar_init(&S.dfull[p], 1);
            bar_init(&S.dempty[p], 4);
        }
        bar_init(&S.drain, 1);
        S.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&S.tmem_base)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;
    bool ok = true;

    auto chunk_cell = [&](int t) -> int64_t { return (first_chunk + t) * kChunk; };
    auto fail = [&]() {
        ok = false;
        *abort_flag = 1;
        atomicExch(status, (int)CNPC_ETIMEOUT);
    };

    if (warp < kConvWarps) {
        // ------------------------------------------------------------ converters
        const int group = warp / 4, q = warp % 4;
        const int L = 32 * q + lane;           // TMEM lane = A' row
        const int hi_half = L < 64;
        const int i = hi_half ? L : L - 64;    // A row
        const bool isA = i < P.na;
        const int j = hi_half ? L - kMaxRowsTc : L - 64 - kMaxRowsTc;  // B row (lanes 40..63, 104..127)
        const bool isB = !isA && i >= kMaxRowsTc && j < P.nb;
        const float *row = isA ? fields + (int64_t)P.a_slot[i] * P.stride
                               : (isB ? fields + (int64_t)P.b_slot[j] * P.stride : nullptr);
        const int gi = isA ? P.a_g[i] : 0;
        const int nrow = hi_half ? j : kMaxColsTc + j;  // B' row of a B lane
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        float4 cur[8], nxt[8];
        auto load = [&](float4 *v, int t) {
            const int64_t c0 = chunk_cell(t);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int64_t c = c0 + 4 * k;
                v[k] = (row && t < nchunk && c < P.ncell) ? __ldg(reinterpret_cast<const float4 *>(row + c))
                                                          : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        load(cur, group);
        load(nxt, group + kGroups);
        for (int t = group; t < nchunk; t += kGroups) {
            const int s = t % kStages;
            // the stage's previous MMAs are done and its weight chunk has landed;
            // the outcome is made warp-uniform before the warp-collective TMEM store
            bool w = t < kStages ||
                     bar_wait(&S.empty[s], (uint32_t)((t / kStages - 1) & 1), P.wait_limit, abort_flag);
            w = w && bar_wait(&S.gfull[t % kGRing], (uint32_t)((t / kGRing) & 1), P.wait_limit, abort_flag);
            if (!__all_sync(0xffffffffu, w)) {
                fail();
                break;
            }
            const int64_t c0 = chunk_cell(t);
            // two halves of 16 cells: A lanes store their values into TMEM (lanes
            // without an A row store zeros; their D rows are never read), B lanes
            // into the shared-memory B' stage
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t out[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) out[k] = 0u;
                if (isA) {
                    const float *gs = gring + ((t % kGRing) * kMaxGs + gi) * kChunk;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const int k = 4 * h + kk;
                        // cells past ncell: zero (the ring slot there holds no weight data)
                        const bool in = c0 + 4 * k < P.ncell;
                        const float4 g4 =
                            in ? *reinterpret_cast<const float4 *>(gs + 4 * k) : make_float4(0.f, 0.f, 0.f, 0.f);
                        const float y[4] = {g4.x * cur[k].x, g4.y * cur[k].y, g4.z * cur[k].z, g4.w * cur[k].w};
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float hv = split_hi(y[e]);
                            out[4 * kk + e] = __float_as_uint(hi_half ? hv : __fsub_rn(y[e], hv));
                        }
                    }
                } else if (isB) {
                    // B' row nrow, 16-byte chunk k at position k ^ (nrow % 8) of its 128-byte row
                    unsigned char *rb = bstage + s * kBStage + (nrow >> 3) * 1024 + (nrow & 7) * 128;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const int k = 4 * h + kk;
                        const float x[4] = {cur[k].x, cur[k].y, cur[k].z, cur[k].w};
                        uint4 w4;
                        uint32_t *wp = reinterpret_cast<uint32_t *>(&w4);
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float hv = split_hi(x[e]);
                            wp[e] = __float_as_uint(hi_half ? hv : __fsub_rn(x[e], hv));
                        }
                        *reinterpret_cast<uint4 *>(rb + ((k ^ (nrow & 7)) << 4)) = w4;
                    }
                }
                __syncwarp();
                tmem_st16(tmem + lane_base + (uint32_t)(kACol0 + kChunk * s + 16 * h), out);
            }
            tmem_wait_st();
            if (isB) proxy_fence();  // B' stores -> tensor-core (async proxy) reads
            tc_fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&S.full[s]);
#pragma unroll
            for (int k = 0; k < 8; ++k) cur[k] = nxt[k];
            load(nxt, t + 2 * kGroups);
            // the 128-byte line of this row kPrefetch chunks ahead (hi-row and
            // B lanes; the lo lanes read the same rows)
            if (row && hi_half && t + kPrefetch < nchunk)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(row + chunk_cell(t + kPrefetch)));
            if (L < P.ngs && t + kPrefetch < nchunk)  // lanes 0..ngs-1 of the group: the weight fields
                asm volatile("prefetch.global.L2 [%0];" ::"l"(P.g[L] + chunk_cell(t + kPrefetch)));
        }
    } else if (warp < kFoldWarp0 + 4) {
        // ------------------------------------------------------------ fold
        const int q = warp - kFoldWarp0;
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        double acc[kMaxColsTc];
#pragma unroll
        for (int c = 0; c < kMaxColsTc; ++c) acc[c] = 0.0;
        const int nper = (nchunk + kPeriod - 1) / kPeriod;
        for (int per = 0; per < nper; ++per) {
            const int p = per & 1;
            const bool w = bar_wait(&S.dfull[p], (uint32_t)((per >> 1) & 1), P.wait_limit, abort_flag);
            if (!__all_sync(0xffffffffu, w)) {  // uniform before the warp-collective TMEM loads
                fail();
                break;
            }
            tc_fence_after();
            float v[kN];
#pragma unroll
            for (int c = 0; c < kN; c += 16) tmem_ld16(tmem + lane_base + (uint32_t)(kDCol * p + c), v + c);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < kMaxColsTc; ++c) acc[c] += (double)(v[c] + v[kMaxColsTc + c]);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&S.dempty[p]);
        }
        ok = __all_sync(0xffffffffu, ok) && !*abort_flag;
        const int L = 32 * q + lane;
        double *dst = partial + ((int64_t)blockIdx.x * 128 + L) * kMaxColsTc;
        const double nanv = __longlong_as_double(0x7ff8000000000000ll);
#pragma unroll
        for (int c = 0; c < kMaxColsTc; ++c) dst[c] = ok ? acc[c] : nanv;
    } else if (lane == 0) {
        // ------------------------------------------------------------ MMA + weight copies
        const uint32_t idesc = idesc_tf32(128, kN);
        int g_issued = 0;  // chunks whose weight copies were issued
        auto issue_g = [&](int t) {
            const int s = t % kGRing;
            const int64_t c0 = chunk_cell(t);
            const int valid = (int)min((int64_t)kChunk, P.ncell - c0);
            const uint32_t bytes = (uint32_t)valid * 4u;
            bar_expect_tx(&S.gfull[s], bytes * (uint32_t)P.ngs);
            for (int gidx = 0; gidx < P.ngs; ++gidx)
                bulk_g2s(gring + (s * kMaxGs + gidx) * kChunk, P.g[gidx] + c0, bytes, &S.gfull[s]);
        };
        for (; g_issued < min(nchunk, kGRing); ++g_issued) issue_g(g_issued);
        int t = 0;
        bool any_mma = false;
        for (; t < nchunk && ok; ++t) {
            const int s = t % kStages;
            const int per = t / kPeriod, p = per & 1;
            const bool first = (t % kPeriod) == 0;
            if (first && per >= 2 &&
                !bar_wait(&S.dempty[p], (uint32_t)(((per >> 1) - 1) & 1), P.wait_limit, abort_flag)) {
                fail();
                break;
            }
            if (!bar_wait(&S.full[s], (uint32_t)((t / kStages) & 1), P.wait_limit, abort_flag)) {
                fail();
                break;
            }
            tc_fence_after();
            const uint32_t bbase = saddr(bstage + s * kBStage);
#pragma unroll
            for (int ks = 0; ks < kChunk / 8; ++ks)
                mma_tf32_ts(tmem + (uint32_t)(kDCol * p), tmem + (uint32_t)(kACol0 + kChunk * s + 8 * ks),
                            umma_desc(bbase + 32 * ks), idesc, (first && ks == 0) ? 0u : 1u);
            any_mma = true;
            mma_commit(&S.empty[s]);
            if ((t % kPeriod) == kPeriod - 1 || t == nchunk - 1) mma_commit(&S.dfull[p]);
            // the converters of chunk t have read its weights: refill its ring slot
            // with chunk t + kGRing
            if (g_issued < nchunk) issue_g(g_issued++);
        }
        // drain: no MMA or copy of this CTA may be in flight when TMEM is freed
        // or the CTA exits
        if (any_mma) {
            mma_commit(&S.drain);
            bar_wait(&S.drain, 0u, kDrainLimit, nullptr);
        }
        for (int u = max(0, g_issued - kGRing); u < g_issued; ++u)
            bar_wait(&S.gfull[u % kGRing], (uint32_t)((u / kGRing) & 1), kDrainLimit, nullptr);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// out[i * nb + j] = sum over blocks of the four TF32 products of (i, j): the
// hi row i and lo row 64 + i of each block's partials, one warp per output,
// fixed order
__global__ void gram_tc_reduce_kernel(const double *partial, int nblocks, int na, int nb, double *out) {
    const int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= na * nb) return;
    const int i = o / nb, j = o % nb;
    double s = 0.0;
    for (int p = lane; p < nblocks; p += 32) {
        const double *blk = partial + (int64_t)p * 128 * kMaxColsTc;
        s += blk[i * kMaxColsTc + j] + blk[(64 + i) * kMaxColsTc + j];
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) out[o] = s;
}

static size_t smem_bytes() {
    return 1024 + (size_t)kStages * kBStage + sizeof(float) * kGRing * kMaxGs * kChunk + sizeof(TcShared);
}

}  // namespace tc

static int run_gram_tc(cnpc_ctx *ctx, int64_t ncell, const float *const *gs, int ngs, const float *fields,
                       int64_t stride, const int *a, const int *ag, int na, const int *b, int nb, double *out,
                       cudaStream_t s) {
    CNPC_REQUIRE(ctx, na >= 1 && na <= tc::kMaxRowsTc && nb >= 1 && nb <= tc::kMaxColsTc,
                 "tensor-core Gram covers 1..40 rows x 1..24 columns");
    CNPC_REQUIRE(ctx, ngs >= 1 && ngs <= tc::kMaxGs, "1..4 weight fields");
    CNPC_REQUIRE(ctx, ncell > 0 && ncell % 4 == 0 && stride >= ncell && stride % 4 == 0,
                 "ncell and field_stride must be positive multiples of 4, field_stride >= ncell");
    CNPC_REQUIRE(ctx, (uintptr_t)fields % 16 == 0, "fields must be 16-byte aligned");
    tc::TcParams P;
    std::memset(&P, 0, sizeof(P));
    P.na = na;
    P.nb = nb;
    P.ngs = ngs;
    P.ncell = ncell;
    P.stride = stride;
    P.wait_limit = ctx->wait_limit;
    for (int k = 0; k < ngs; ++k) {
        CNPC_REQUIRE(ctx, gs[k] != nullptr && (uintptr_t)gs[k] % 16 == 0, "weight fields must be 16-byte aligned");
        P.g[k] = gs[k];
    }
    for (int i = 0; i < na; ++i) {
        CNPC_REQUIRE(ctx, a[i] >= 0, "negative field index");
        CNPC_REQUIRE(ctx, ag[i] >= 0 && ag[i] < ngs, "row weight index out of range");
        P.a_slot[i] = a[i];
        P.a_g[i] = ag[i];
    }
    for (int j = 0; j < nb; ++j) {
        CNPC_REQUIRE(ctx, b[j] >= 0, "negative field index");
        P.b_slot[j] = b[j];
    }
    const int64_t nchunks = (ncell + tc::kChunk - 1) / tc::kChunk;
    const int nblocks = (int)std::min<int64_t>(ctx->num_sms, nchunks);
    const size_t part_bytes = (size_t)nblocks * 128 * tc::kMaxColsTc * sizeof(double);
    int st = ensure_scratch(ctx, part_bytes, s);
    if (st) return st;
    st = ensure_status(ctx);
    if (st) return st;
    double *part = (double *)ctx->scratch;
    const size_t smem = tc::smem_bytes();
    st = check_cuda(ctx, cudaFuncSetAttribute(tc::gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem), "gram_tc_kernel smem");
    if (st) return st;
    tc::gram_tc_kernel<<<nblocks, tc::kThreads, smem, s>>>(fields, P, part, ctx->d_status);
    st = check_launch(ctx, "gram_tc_kernel");
    if (st) return st;
    const int nout = na * nb;
    tc::gram_tc_reduce_kernel<<<(nout + 7) / 8, 256, 0, s>>>(part, nblocks, na, nb, out);
    return check_launch(ctx, "gram_tc_reduce_kernel");
}

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_contract_gram_tc(cnpc_ctx *ctx, int64_t ncell, const float *d_g, const float *d_fields,
                                     int64_t field_stride, const int *h_a, int na, const int *h_b, int nb,
                                     double *d_out, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, d_g && d_fields && d_out && h_a && h_b, "null argument");
    CNPC_REQUIRE(ctx, na >= 1 && na <= tc::kMaxRowsTc, "tensor-core Gram covers 1..40 rows x 1..24 columns");
    int ag[tc::kMaxRowsTc] = {0};
    const float *gs[1] = {d_g};
    return run_gram_tc(ctx, ncell, gs, 1, d_fields, field_stride, h_a, ag, na, h_b, nb, d_out,
                       (cudaStream_t)stream);
}

extern "C" int cnpc_contract_gram_tc_multi_g(cnpc_ctx *ctx, int64_t ncell, const float *const *h_gs, int ngs,
                                             const float *d_fields, int64_t field_stride, const int *h_a,
                                             const int *h_ag, int na, const int *h_b, int nb, double *d_out,
                                             cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, h_gs && d_fields && d_out && h_a && h_ag && h_b, "null argument");
    return run_gram_tc(ctx, ncell, h_gs, ngs, d_fields, field_stride, h_a, h_ag, na, h_b, nb, d_out,
                       (cudaStream_t)stream);
}
