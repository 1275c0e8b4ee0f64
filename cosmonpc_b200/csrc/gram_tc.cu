// FP32 Gram contraction on the 5th-generation tensor cores (tcgen05, TF32 pairs).
//
//   out[i][j] = sum_x G_{g_i}(x) F_{a_i}(x) F_{b_j}(x),  i < na <= 40, j < nb <= 24
//
// is a GEMM D = A B^T with rows A_i = G_{g_i} F_{a_i}, columns B_j = F_{b_j} and
// K = cells.  Each FP32 operand y is split into a TF32 pair y = hi + lo: hi is
// y rounded to 11 significant bits (integer add of half a TF32 unit to the
// magnitude bits, a carry moving into the exponent as rounding requires; the
// tensor core reads an FP32 bit pattern as TF32 by dropping the low 13 bits,
// measured, so hi is stored as that sum), lo = y - hi exactly (Sterbenz),
// |lo| <= 2^-12 |y|, and the tensor core's TF32 view of lo drops at most
// 2^-23 |y|.  ONE MMA per K-step of 8 cells takes all four products:
// A' = [A_hi ; A_lo] (M = 128: rows 0..39 hi, 64..103 lo), B' = [B_hi ; B_lo]
// (N = 48: rows 0..23 hi, 24..47 lo), so
//   C[i][j] = D[i][j] + D[i][24+j] + D[64+i][j] + D[64+i][24+j].
// A' lives in tensor memory (the MMA's A-from-TMEM form), B' in 128-byte
// swizzled K-major shared memory.
//
// A CTA per SM walks a contiguous run of stages of 128 cells (4 K-blocks of 32
// cells).  Warp roles:
//   * producer warp: copies the stage's 128 cells of every staged row (the
//     distinct rows of A, B and the weight fields, at most 68) with one warp
//     instruction of 16-byte cp.async each into a raw ring of as many stages
//     as shared memory holds (<= 8); rows are padded by 16 bytes so that lanes
//     reading different rows at the same cell hit different banks.  (One
//     cp.async.bulk of 512 bytes per row and stage ran at ~63 cycles per copy,
//     2.3 TB/s over the GPU.)
//   * two groups of four converter warps (one warp per TMEM lane quarter):
//     group g converts chunk g (cells 64 g .. 64 g + 63) of every stage into
//     one of its three converted slots (TMEM A' + shared B'), so it converts
//     ahead while the MMAs read its earlier slots.  Lane L = 32 q + lane owns
//     A' row L: lanes 0..39 / 64..103 read their field row and weight row,
//     form G F and keep hi / lo; lanes 40..63 / 104..127 take B row L - 40 /
//     L - 104 and keep its hi / lo.  Every lane stores its 32 values of a
//     K-block into TMEM with one tcgen05.st (B lanes' TMEM rows feed D rows
//     that are never read) and B lanes also store them into the slot's B'.
//   * MMA (one thread): 8 MMAs per chunk into one of two accumulator sets,
//     committed to the slot's "converted-empty" barrier; every kPeriod
//     stages the set's completion is committed to the fold warps.
//   * four fold warps read a finished set (tcgen05.ld), add D[L][j] +
//     D[L][24+j] into FP64 registers and release it, so FP32 only ever sums
//     kPeriod * 128 cells of one accumulator.
// Per-CTA FP64 partials are reduced in a fixed order (bitwise reproducible).
//
// Budget per 64 cells and SM: 41 rows x 256 bytes from HBM (~460 cycles at
// the measured copy bandwidth), 8 MMAs (one M = 128, N <= 64 TF32 MMA takes
// 45-54 cycles back to back from one thread, measured with rotating operands,
// commits and concurrent TMEM stores).  Measured at 256^3, 40 x 20 outputs:
// 1.15-1.19 ms, against 0.84 ms for the CUDA-core FFMA kernel, and the same
// with 20 rows: the hand-offs, not the copies, bound it.  An mbarrier
// try_wait costs ~240 cycles even when its phase has completed (one per 8
// MMAs takes them from 54 to 84 cycles each), and every chunk pays one on the
// MMA thread and two on each converter warp; with the converters' arithmetic
// removed (timing copy) the kernel still took 0.91 ms.  Replacing the
// hand-offs to the MMA thread by release / acquire counters in shared memory,
// with the producer warp republishing copy completions, measured 1.23-1.46 ms
// (the republishing adds its own test latency).
//
// Every mbarrier wait is bounded (the context's wait limit): a wait that gives
// up sets the abort flag and the context's status word (CNPC_ETIMEOUT), every
// role stops, the producer and the MMA thread drain their own copies and MMAs
// (bounded by a fixed limit) before TMEM is freed, and the CTA's partials are
// NaN.
#include <algorithm>
#include <cstring>

#include "internal.h"

namespace cnpc {
namespace tc {

constexpr int kCell = 128;                 // cells per stage
constexpr int kKB = kCell / 32;            // K-blocks of 32 cells (one 128-byte swizzle atom of K) per stage
constexpr int kMaxRaw = 8;                 // raw ring depth: as many stages as shared memory holds, <= 8
constexpr int kConvGroups = 2;             // converter warp groups: group g converts chunk g of every stage
constexpr int kChunkKB = kKB / kConvGroups;  // K-blocks per chunk (64 cells)
constexpr int kConvSlots = 6;              // converted chunks (TMEM A' + shared B') in flight, 3 per group
constexpr int kPeriod = 4;                 // stages per accumulator set
constexpr int kMaxRowsTc = 40;
constexpr int kMaxColsTc = 24;
constexpr int kMaxGs = 4;
constexpr int kMaxStaged = kMaxRowsTc + kMaxColsTc + kMaxGs;
constexpr int kRowPitch = kCell + 4;       // floats: 512 bytes + 16 bytes of bank padding
constexpr int kN = 48;                     // B' rows: hi 0..23, lo 24..47
constexpr int kBBlock = kN / 8 * 1024;     // one K-block of B': 6 row groups of 8 rows x 128 bytes
constexpr int kDCol = 64;                  // accumulator set p at TMEM column 64 p
constexpr int kACol0 = 128;                // A' slot s, K-block kb at TMEM column 128 + 64 s + 32 kb
constexpr int kTmemCols = 512;
constexpr int kConvWarp0 = 1;              // warps 1 .. 4 kConvGroups convert
constexpr int kMmaWarp = kConvWarp0 + 4 * kConvGroups;
constexpr int kFoldWarp0 = kMmaWarp + 1;   // four fold warps
constexpr int kThreads = 32 * (kFoldWarp0 + 4);
constexpr int kSmemMax = 227 * 1024;
constexpr long long kDrainLimit = 1ll << 22;
constexpr int kStorePiece = 32;            // TMEM columns per tcgen05.st of a converter lane (8 or 32)
constexpr int kIdleSleepNs = 0;            // back-off of the fold and producer waits (0: spin)
static_assert(kACol0 + kConvSlots * kChunkKB * 32 <= kTmemCols, "TMEM columns");
static_assert(kConvSlots % kConvGroups == 0, "slots per group");

struct TcParams {
    int na, nb, nstaged, nraw;
    int64_t ncell;
    long long wait_limit;
    const float *staged[kMaxStaged];  // staged rows: device addresses of the rows' cell 0
    int a_src[kMaxRowsTc];            // staged row of A row i
    int a_gsrc[kMaxRowsTc];           // staged row of A row i's weight field
    int b_src[kMaxColsTc];            // staged row of B row j
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
// Bounded wait: false after `limit` polls, or as soon as another role aborted;
// sleep_ns > 0 backs off between polls.
__device__ inline bool bar_wait(uint64_t *bar, uint32_t parity, long long limit, volatile int *abort_flag,
                                int sleep_ns = 0) {
    for (long long i = 0; i < limit; ++i) {
        if (bar_try(bar, parity)) return true;
        if (abort_flag && (i & 63) == 63 && *abort_flag) return false;
        if (sleep_ns > 0) __nanosleep(sleep_ns);
    }
    return false;
}

// 16-byte asynchronous copy global -> shared (L1 bypassed)
__device__ inline void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
// arrive on the barrier once this thread's earlier cp.async copies have landed
// (the barrier's expected count includes this arrival)
__device__ inline void cp_async_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(saddr(bar)) : "memory");
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
// 8 consecutive TMEM columns of this thread's lane
__device__ inline void tmem_st8(uint32_t taddr, const uint32_t *v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
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

// One K-block (32 cells) of a converter lane's A' row: y = G x (A lanes) or x
// (B lanes), its TF32 hi (HI) or lo part into the lane's 32 TMEM columns and,
// for B lanes, into B' row brow (16-byte chunk k at k ^ (brow % 8) of the
// row's 128 bytes).  TAIL: the stage ends at vcells (the ring holds stale or
// unwritten data past it), those cells count as zero.  Lanes without a row
// convert row 0 of the stage: their TMEM rows and B' rows feed only D rows and
// columns that are never read.  All shared loads of the K-block are issued
// before the arithmetic.
template <bool HI, bool TAIL>
__device__ __forceinline__ void convert_kblock(const float *xr, const float *gr, bool isA, int kb, int vcells,
                                               unsigned char *rb, int brow, uint32_t taddr) {
    float4 x4[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x4[k] = *reinterpret_cast<const float4 *>(xr + 32 * kb + 4 * k);
    if (isA) {
        float4 g4[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) g4[k] = *reinterpret_cast<const float4 *>(gr + 32 * kb + 4 * k);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float2 a = __fmul2_rn(make_float2(g4[k].x, g4[k].y), make_float2(x4[k].x, x4[k].y));
            const float2 b = __fmul2_rn(make_float2(g4[k].z, g4[k].w), make_float2(x4[k].z, x4[k].w));
            x4[k] = make_float4(a.x, a.y, b.x, b.y);
        }
    }
    uint32_t out[32];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float y[4] = {x4[k].x, x4[k].y, x4[k].z, x4[k].w};
        if (TAIL && 32 * kb + 4 * k >= vcells) y[0] = y[1] = y[2] = y[3] = 0.f;  // vcells is a multiple of 4
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            // hi: the tensor core reads an FP32 pattern as TF32 by dropping the
            // low 13 bits, so y's bits plus half a TF32 unit give hi rounded
            const uint32_t r = __float_as_uint(y[e]) + 0x1000u;
            out[4 * k + e] = HI ? r : __float_as_uint(__fsub_rn(y[e], __uint_as_float(r & 0xFFFFE000u)));
        }
    }
    if (!isA) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            *reinterpret_cast<uint4 *>(rb + ((k ^ (brow & 7)) << 4)) =
                make_uint4(out[4 * k], out[4 * k + 1], out[4 * k + 2], out[4 * k + 3]);
    }
    if (kStorePiece == 32) {
        tmem_st32(taddr, out);
    } else {
#pragma unroll
        for (int c = 0; c < 32; c += 8) tmem_st8(taddr + c, out + c);
    }
}

struct __align__(8) TcShared {
    uint64_t rfull[kMaxRaw];       // a raw stage's copies landed (32 producer lanes, cp.async noinc)
    uint64_t rempty[kMaxRaw];      // the converters have read a raw stage (8 warps)
    uint64_t cfull[kConvSlots];    // a converted slot is written (4 warps)
    uint64_t cempty[kConvSlots];   // a converted slot's MMAs are done (tcgen05.commit)
    uint64_t dfull[2];             // accumulator set complete (tcgen05.commit)
    uint64_t dempty[2];            // accumulator set folded (4 fold warps)
    uint64_t drain;
    uint32_t tmem_base;
    int abort_flag;
};

// 512 in the bounds caps registers at 128 (four warps per scheduler fit)
__global__ void __launch_bounds__(512, 1) gram_tc_kernel(const TcParams P, double *__restrict__ partial,
                                                              int *status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned B' slots, then the raw ring, then the barriers
    unsigned char *base = smem_raw + ((1024 - (saddr(smem_raw) & 1023)) & 1023);
    unsigned char *bconv = base;  // [kConvSlots][kChunkKB][kBBlock]
    float *raw = reinterpret_cast<float *>(base + kConvSlots * kChunkKB * kBBlock);  // [nraw][nstaged][kRowPitch]
    const int raw_stage = P.nstaged * kRowPitch;
    const int nraw = P.nraw;
    TcShared &S = *reinterpret_cast<TcShared *>(raw + nraw * raw_stage);
    volatile int *abort_flag = &S.abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // each CTA takes a contiguous run of stages
    const int64_t nst_all = (P.ncell + kCell - 1) / kCell;
    const int64_t per_cta = (nst_all + gridDim.x - 1) / gridDim.x;
    const int64_t first = (int64_t)blockIdx.x * per_cta;
    const int nst = first < nst_all ? (int)min(per_cta, nst_all - first) : 0;
    const int nch = kConvGroups * nst;  // converted chunks

    if (threadIdx.x == 0) {
        for (int r = 0; r < nraw; ++r) {
            bar_init(&S.rfull[r], 32);
            bar_init(&S.rempty[r], 4 * kConvGroups);
        }
        for (int c = 0; c < kConvSlots; ++c) {
            bar_init(&S.cfull[c], 4);
            bar_init(&S.cempty[c], 1);
        }
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
    auto fail = [&]() {
        ok = false;
        *abort_flag = 1;
        atomicExch(status, (int)CNPC_ETIMEOUT);
    };

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        // lane l copies cells 4 l .. 4 l + 3 of every staged row (one 512-byte
        // row per warp instruction); each lane's arrival on the stage's barrier
        // fires when its own copies have landed
        for (int t = 0; t < nst; ++t) {
            const int r = t % nraw;
            const bool w = t < nraw || bar_wait(&S.rempty[r], (uint32_t)((t / nraw - 1) & 1), P.wait_limit, abort_flag,
                                                kIdleSleepNs);
            if (!__all_sync(0xffffffffu, w)) {
                fail();
                break;
            }
            const int64_t c0 = (first + t) * kCell;
            const int vcells = (int)min((int64_t)kCell, P.ncell - c0);
            float *dst = raw + r * raw_stage + 4 * lane;
            if (4 * lane < vcells)
                for (int u = 0; u < P.nstaged; ++u) cp_async16(dst + u * kRowPitch, P.staged[u] + c0 + 4 * lane);
            cp_async_arrive_noinc(&S.rfull[r]);
        }
        // no copy may be in flight when the CTA exits
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp < kMmaWarp) {
        // ------------------------------------------------------------ converters
        const int group = (warp - kConvWarp0) / 4;  // converts cells 64 group .. of every stage
        const int q = warp & 3;            // the TMEM lane quarter this warp may access
        const int L = 32 * q + lane;       // A' row
        const bool hi = L < 64;            // warp-uniform
        const int i = L & 63;
        const bool isA = i < kMaxRowsTc;   // else B row j
        const int j = i - kMaxRowsTc;
        const bool valid = isA ? i < P.na : j < P.nb;
        const int src = valid ? (isA ? P.a_src[i] : P.b_src[j]) : 0;
        const int gsrc = valid && isA ? P.a_gsrc[i] : 0;
        const int brow = hi ? j : kMaxColsTc + j;  // B' row of a B lane
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        for (int t = 0; t < nst; ++t) {
            const int h = kConvGroups * t + group;  // chunk index
            const int r = t % nraw, sl = h % kConvSlots;
            // the raw stage has landed and the slot's previous MMAs are done; the
            // outcome is made warp-uniform before the warp-collective TMEM stores
            bool w = bar_wait(&S.rfull[r], (uint32_t)((t / nraw) & 1), P.wait_limit, abort_flag);
            w = w && (h < kConvSlots ||
                      bar_wait(&S.cempty[sl], (uint32_t)((h / kConvSlots - 1) & 1), P.wait_limit, abort_flag));
            if (!__all_sync(0xffffffffu, w)) {
                fail();
                break;
            }
            tc_fence_after();
            const int vcells = (int)min((int64_t)kCell, P.ncell - (first + t) * kCell);
            const bool tail = vcells < kCell;  // warp-uniform, like hi
            const float *xr = raw + r * raw_stage + src * kRowPitch;
            const float *gr = raw + r * raw_stage + gsrc * kRowPitch;
#pragma unroll 1
            for (int u = 0; u < kChunkKB; ++u) {
                const int kb = group * kChunkKB + u;  // K-block of the stage
                unsigned char *rb = bconv + (sl * kChunkKB + u) * kBBlock + (brow >> 3) * 1024 + (brow & 7) * 128;
                const uint32_t ta = tmem + lane_base + (uint32_t)(kACol0 + sl * kChunkKB * 32 + u * 32);
                if (hi) {
                    if (tail) convert_kblock<true, true>(xr, gr, isA, kb, vcells, rb, brow, ta);
                    else convert_kblock<true, false>(xr, gr, isA, kb, vcells, rb, brow, ta);
                } else {
                    if (tail) convert_kblock<false, true>(xr, gr, isA, kb, vcells, rb, brow, ta);
                    else convert_kblock<false, false>(xr, gr, isA, kb, vcells, rb, brow, ta);
                }
            }
            tmem_wait_st();
            if (!isA) proxy_fence();  // B' stores -> tensor-core (async proxy) reads
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                bar_arrive(&S.rempty[r]);
                bar_arrive(&S.cfull[sl]);
            }
        }
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------------------ MMA
        if (lane == 0) {
            // a single thread's instruction latency between MMAs sets the issue
            // rate (one M = 128, N = 48 MMA takes 46.5 cycles back to back), so
            // descriptors advance by constant adds and the rings by counters
            const uint32_t idesc = idesc_tf32(128, kN);
            const uint64_t desc0 = umma_desc(saddr(bconv));  // + 16-byte units of B' offset
            constexpr int kPeriodCh = kPeriod * kConvGroups;  // chunks per accumulator set
            bool any_mma = false;
            int sl = 0, use = 0, pc = 0, per = 0;  // slot, its use count, chunk in period, period
            for (int h = 0; h < nch; ++h) {
                const int p = per & 1;
                if (pc == 0 && per >= 2 &&
                    !bar_wait(&S.dempty[p], (uint32_t)(((per >> 1) - 1) & 1), P.wait_limit, abort_flag)) {
                    fail();
                    break;
                }
                if (!bar_wait(&S.cfull[sl], (uint32_t)(use & 1), P.wait_limit, abort_flag)) {
                    fail();
                    break;
                }
                tc_fence_after();
                const uint32_t d_t = tmem + (uint32_t)(kDCol * p);
                const uint32_t a_t = tmem + (uint32_t)(kACol0 + sl * kChunkKB * 32);
                const uint64_t b_d = desc0 + (uint64_t)(sl * kChunkKB * (kBBlock >> 4));
                mma_tf32_ts(d_t, a_t, b_d, idesc, pc == 0 ? 0u : 1u);
#pragma unroll
                for (int m = 1; m < kChunkKB * 4; ++m)  // K-block m / 4, K-step m % 4
                    mma_tf32_ts(d_t, a_t + (uint32_t)(8 * m), b_d + (uint64_t)((m >> 2) * (kBBlock >> 4) + 2 * (m & 3)),
                                idesc, 1u);
                any_mma = true;
                mma_commit(&S.cempty[sl]);
                if (pc == kPeriodCh - 1 || h == nch - 1) mma_commit(&S.dfull[p]);
                if (++sl == kConvSlots) {
                    sl = 0;
                    ++use;
                }
                if (++pc == kPeriodCh) {
                    pc = 0;
                    ++per;
                }
            }
            // no MMA of this CTA may be in flight when TMEM is freed
            if (any_mma) {
                mma_commit(&S.drain);
                bar_wait(&S.drain, 0u, kDrainLimit, nullptr);
            }
        }
    } else if (warp >= kFoldWarp0) {
        // ------------------------------------------------------------ fold
        const int q = warp & 3;
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        double acc[kMaxColsTc];
#pragma unroll
        for (int c = 0; c < kMaxColsTc; ++c) acc[c] = 0.0;
        const int nper = (nst + kPeriod - 1) / kPeriod;
        for (int per = 0; per < nper; ++per) {
            const int p = per & 1;
            const bool w = bar_wait(&S.dfull[p], (uint32_t)((per >> 1) & 1), P.wait_limit, abort_flag, kIdleSleepNs);
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
            for (int c = 0; c < kMaxColsTc; ++c) acc[c] += (double)v[c] + (double)v[kMaxColsTc + c];
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

static size_t smem_fixed() { return 1024 + (size_t)kConvSlots * kChunkKB * kBBlock + sizeof(TcShared); }
static size_t raw_stage_bytes(int nstaged) { return sizeof(float) * (size_t)nstaged * kRowPitch; }

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
    P.ncell = ncell;
    P.wait_limit = ctx->wait_limit;
    // staged rows: every distinct field row of A and B, then the weight fields
    auto stage_row = [&](const float *ptr) -> int {
        for (int u = 0; u < P.nstaged; ++u)
            if (P.staged[u] == ptr) return u;
        P.staged[P.nstaged] = ptr;
        return P.nstaged++;
    };
    for (int i = 0; i < na; ++i) {
        CNPC_REQUIRE(ctx, a[i] >= 0, "negative field index");
        CNPC_REQUIRE(ctx, ag[i] >= 0 && ag[i] < ngs, "row weight index out of range");
        P.a_src[i] = stage_row(fields + (int64_t)a[i] * stride);
    }
    for (int j = 0; j < nb; ++j) {
        CNPC_REQUIRE(ctx, b[j] >= 0, "negative field index");
        P.b_src[j] = stage_row(fields + (int64_t)b[j] * stride);
    }
    int gsrc[tc::kMaxGs];
    for (int k = 0; k < ngs; ++k) {
        CNPC_REQUIRE(ctx, gs[k] != nullptr && (uintptr_t)gs[k] % 16 == 0, "weight fields must be 16-byte aligned");
        gsrc[k] = stage_row(gs[k]);
    }
    for (int i = 0; i < na; ++i) P.a_gsrc[i] = gsrc[ag[i]];
    const int64_t nstages = (ncell + tc::kCell - 1) / tc::kCell;
    const int nblocks = (int)std::min<int64_t>(ctx->num_sms, nstages);
    const size_t part_bytes = (size_t)nblocks * 128 * tc::kMaxColsTc * sizeof(double);
    int st = ensure_scratch(ctx, part_bytes, s);
    if (st) return st;
    st = ensure_status(ctx);
    if (st) return st;
    double *part = (double *)ctx->scratch;
    // as many raw stages as the shared memory holds (>= 2 for <= 68 staged rows)
    P.nraw = (int)std::min<size_t>(tc::kMaxRaw, (tc::kSmemMax - tc::smem_fixed()) / tc::raw_stage_bytes(P.nstaged));
    CNPC_REQUIRE(ctx, P.nraw >= 2, "tensor-core Gram: too many staged rows");
    const size_t smem = tc::smem_fixed() + (size_t)P.nraw * tc::raw_stage_bytes(P.nstaged);
    st = check_cuda(ctx, cudaFuncSetAttribute(tc::gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem), "gram_tc_kernel smem");
    if (st) return st;
    tc::gram_tc_kernel<<<nblocks, tc::kThreads, smem, s>>>(P, part, ctx->d_status);
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
