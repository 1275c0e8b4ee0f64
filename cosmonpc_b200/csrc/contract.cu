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
// the current one is contracted.  Every mbarrier wait is bounded (the
// context's wait limit, in polls): a wait that gives up records CNPC_ETIMEOUT
// in the status word, the block drains its own copies (bounded by the fixed
// kWaitLimit, so that no copy is in flight when the block exits) and its
// outputs become NaN.
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

constexpr int kMaxRows = 128;
constexpr int kMaxUnion = 264;
constexpr long long kWaitLimit = 1ll << 22;  // try_wait polls before giving up (~seconds)


struct GramParams {
    int na, nb, nunion, ncopy, g_row, ct, ntiles, ngroups, flush_chunks, nstages;
    int64_t ncell, field_stride;
    long long wait_limit;  // polls of a pipeline wait before it gives up
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
// Bounded wait; returns false if the barrier phase did not complete within
// `limit` polls (0: give up at once).
__device__ inline bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit = kWaitLimit) {
    for (long long i = 0; i < limit; ++i)
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

constexpr int kMaxStages = 4;

// Chunk (cells per staged row) is a compile-time constant so that every
// shared-memory operand offset in the inner loop is an immediate.
template <typename T> struct ChunkOf;
template <> struct ChunkOf<float> { static constexpr int C = 256; };
template <> struct ChunkOf<double> { static constexpr int C = 128; };

// Block group g owns tiles [16g, 16g + nt); warp w works on tile 16g + (w % nt)
// and, when several warps share a tile, takes every nphase-th slice of cells.
struct WarpWork {
    int tile, phase, nphase;
};
__device__ inline WarpWork warp_work(int group, int warp, int nwarps, int ntiles) {
    const int t0 = group * nwarps;
    const int nt = min(nwarps, ntiles - t0);
    WarpWork w;
    w.tile = t0 + warp % nt;
    w.phase = warp / nt;
    w.nphase = (nwarps - 1 - warp % nt) / nt + 1;
    return w;
}

// FP64 tile step: one cell per lane, 8x4 accumulators in FP64.
struct Fp64Tile {
    static constexpr int TM = 8, TN = 4, NV = 32, WARPS = 16, CHUNK = 128;
    double acc[TM][TN];
    __device__ void zero() {
#pragma unroll
        for (int r = 0; r < TM; ++r)
#pragma unroll
            for (int q = 0; q < TN; ++q) acc[r][q] = 0.0;
    }
    __device__ void step(const double *rowG, const double *rowA, const double *rowB, int c) {
        const double gv = rowG[c];
        double av[TM], bv[TN];
#pragma unroll
        for (int r = 0; r < TM; ++r) av[r] = gv * rowA[r * CHUNK + c];
#pragma unroll
        for (int q = 0; q < TN; ++q) bv[q] = rowB[q * CHUNK + c];
#pragma unroll
        for (int r = 0; r < TM; ++r)
#pragma unroll
            for (int q = 0; q < TN; ++q) acc[r][q] = fma(av[r], bv[q], acc[r][q]);
    }
    __device__ void fold(double *acc64, int lane) {
        double v[NV];
#pragma unroll
        for (int r = 0; r < TM; ++r)
#pragma unroll
            for (int q = 0; q < TN; ++q) v[r * TN + q] = acc[r][q];
        TransposeReduce<double, NV, 16>::run(v, lane);
        acc64[0] += v[0];
        zero();
    }
};

template <typename T> struct TileOf;
template <> struct TileOf<double> { using type = Fp64Tile; };

template <typename T, int NWARPS>
__global__ void __launch_bounds__(NWARPS * 32, 1)
    gram_kernel(const T *__restrict__ g, const T *__restrict__ fields, const GramParams P, double *partial,
                int *status) {
    using Tile = typename TileOf<T>::type;
    constexpr int TM = Tile::TM, TN = Tile::TN, NV = Tile::NV, NW = Tile::WARPS, CHUNK = Tile::CHUNK;
    constexpr int CPL = sizeof(T) == 4 ? 2 : 1;  // cells per lane per step
    constexpr int PER_LANE = NV / 32;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kMaxStages];
    __shared__ __align__(8) uint64_t empty_bar[kMaxStages];
    __shared__ volatile int abort_flag;
    const int NST = P.nstages;
    const int nf = P.nunion;  // staged rows (G, A rows, separate B rows), see run_gram
    const int stage_elems = nf * CHUNK;
    T *const stage0 = reinterpret_cast<T *>(smem_raw);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int group = blockIdx.x % P.ngroups;
    const int xr = blockIdx.x / P.ngroups;
    const int nxr = gridDim.x / P.ngroups;
    const WarpWork ww = warp_work(group, warp, NW, P.ntiles);
    const int a_row = P.a_slot[(ww.tile / P.ct) * TM];   // first staged row of this tile's A rows
    const int b_row = P.b_slot[(ww.tile % P.ct) * TN];   // first staged row of its B rows

    Tile tile;
    tile.zero();
    double acc64[PER_LANE];
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) acc64[e] = 0.0;

    const int64_t first = (int64_t)xr * CHUNK;
    const int64_t step = (int64_t)nxr * CHUNK;
    const int nchunk = first < P.ncell ? (int)((P.ncell - first + step - 1) / step) : 0;
    const bool producer = threadIdx.x == 0;

    auto issue = [&](int k) {  // bulk copies of this block's k-th chunk
        const int s = k % NST;
        const int64_t c0 = first + (int64_t)k * step;
        const int64_t valid = min((int64_t)CHUNK, P.ncell - c0);
        const uint32_t bytes = (uint32_t)(valid * sizeof(T));
        T *dst = stage0 + s * stage_elems;
        fence_proxy_async();
        mbar_expect_tx(&full_bar[s], bytes * (uint32_t)P.ncopy);
        for (int u = 0; u < nf; ++u) {
            const int f = P.union_field[u];
            if (f == -1) continue;  // padding row: never read into a kept output
            const T *src = f == -2 ? g + c0 : fields + (int64_t)f * P.field_stride + c0;
            bulk_g2s(dst + u * CHUNK, src, bytes, &full_bar[s]);
        }
    };

    if (producer) {
        abort_flag = 0;
        for (int s = 0; s < NST; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], NW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = 0;
    if (producer)
        for (; issued < min(nchunk, NST - 1); ++issued) issue(issued);

    int since_flush = 0;
    int k = 0;
    for (; k < nchunk; ++k) {
        const int s = k % NST;
        if (producer && issued < nchunk && !abort_flag) {
            const int sp = issued % NST;
            if (issued >= NST &&
                !mbar_wait_bounded(&empty_bar[sp], (uint32_t)(((issued / NST) - 1) & 1), P.wait_limit)) {
                abort_flag = 1;
                atomicExch(status, (int)CNPC_ETIMEOUT);
            } else {
                issue(issued);
                ++issued;
            }
        }
        if (!mbar_wait_bounded(&full_bar[s], (uint32_t)((k / NST) & 1), P.wait_limit)) {
            abort_flag = 1;
            if (lane == 0) atomicExch(status, (int)CNPC_ETIMEOUT);
        }
        if (abort_flag) break;
        const T *sb = stage0 + s * stage_elems;
        const int valid = (int)min((int64_t)CHUNK, P.ncell - (first + (int64_t)k * step));
        const T *rowG = sb + P.g_row * CHUNK;
        const T *rowA = sb + a_row * CHUNK;
        const T *rowB = sb + b_row * CHUNK;
        for (int c = CPL * (lane + 32 * ww.phase); c < valid; c += CPL * 32 * ww.nphase)
            tile.step(rowG, rowA, rowB, c);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[s]);
        if (++since_flush == P.flush_chunks) {
            since_flush = 0;
            tile.fold(acc64, lane);
        }
    }
    if (abort_flag && producer) {
        for (int j = k; j < issued; ++j) mbar_wait_bounded(&full_bar[j % NST], (uint32_t)((j / NST) & 1));
    }
    tile.fold(acc64, lane);
    double *dst = partial + ((int64_t)blockIdx.x * NW + warp) * NV;
    const double nanv = __longlong_as_double(0x7ff8000000000000ll);
    const bool bad = abort_flag != 0;
#pragma unroll
    for (int e = 0; e < PER_LANE; ++e) dst[lane * PER_LANE + e] = bad ? nanv : acc64[e];
}


// ---------------------------------------------------------------------------
// FP32 fields.  Every warp is independent: it owns a (8 RB) x (4 CB) output
// window for a 32-cell slab of each block chunk, streams that slab of every
// staged row with 16-byte cp.async into a private double-buffered shared-memory
// tile (rows padded to 36 floats), and contracts the previous slab meanwhile.
// Lane (g, h) = (lane / 4, lane % 4) owns rows g + 8 r and columns h + 4 q, so a
// shared-memory load of one row is either a broadcast or hits 8 distinct
// banks.  Two adjacent cells are read per 8-byte load and accumulated with
// packed FP32x2 FMAs (even and odd cell partial sums); the FP32 partials are
// folded into this warp's FP64 partials (in L2) every kFfFold chunks.
constexpr int kFfWarps = 8;
constexpr int kFfChunk = 256;  // cells per block chunk (32 per warp)
constexpr int kFfRow = 36;     // padded slab row (32 cells + 4)
// chunks per FP32 partial: 16 (512 cells per lane); each fold is a dependent
// read-modify-write of the L2-resident FP64 partials, and folding every 4 / 8 /
// 16 chunks took the 40 x 20 launch at 256^3 to 0.848 / 0.813 / 0.797 ms
constexpr int kFfFold = 16;
constexpr int kFfMaxRows = 80;  // staged rows: <= 4 weights + 48 A + 24 B
constexpr int kFfTable = kFfMaxRows * 8;  // bytes of the row-source table ahead of the slabs

__device__ inline void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ inline void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Several weight fields in one launch (MG): staged rows [G_0 .. G_{k-1}][A][B],
// window row i multiplied by G_{grow[i]}; union_field -2 - j names G_j.
struct FfMulti {
    const float *g[4];
    int grow[48];
};

template <int RB, int CB, int NBUF, bool MG>
__global__ void __launch_bounds__(kFfWarps * 32, 2)
    gram_ffma_kernel(const float *__restrict__ g, const float *__restrict__ fields, const GramParams P,
                     const FfMulti X, double *partial) {
    constexpr int WR = 8 * RB, WC = 4 * CB;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nrows = P.nunion;  // staged rows: G, A window, separate B window
    const int slab = nrows * kFfRow;
    // the block's table of staged-row sources (nullptr: padding row), then the slabs
    const float **rowsrc = reinterpret_cast<const float **>(smem_raw);
    float *const buf0 = reinterpret_cast<float *>(smem_raw + kFfTable) + (size_t)warp * NBUF * slab;
    const int64_t nchunk_all = (P.ncell + kFfChunk - 1) / kFfChunk;
    const int nchunk = blockIdx.x < nchunk_all ? (int)((nchunk_all - 1 - blockIdx.x) / gridDim.x + 1) : 0;
    for (int u = threadIdx.x; u < nrows; u += blockDim.x) {
        const int f = P.union_field[u];
        rowsrc[u] = f >= 0 ? fields + (int64_t)f * P.field_stride : (f == -1 ? nullptr : (MG ? X.g[-2 - f] : g));
    }
    __syncthreads();

    // stream this warp's 32-cell slab of chunk k into buffer b: lane l copies
    // the 16 bytes (l % 8) of rows l / 8 + 4 j
    const int part = lane & 7, row0 = lane >> 3;
    auto issue = [&](int k, int b) {
        const int64_t cell = ((int64_t)blockIdx.x + (int64_t)k * gridDim.x) * kFfChunk + warp * 32 + part * 4;
        float *d = buf0 + b * slab + row0 * kFfRow + part * 4;
        if (cell < P.ncell) {  // ncell is a multiple of 4, so the 16 bytes are all valid
            for (int row = row0; row < nrows; row += 4, d += 4 * kFfRow) {
                const float *src = rowsrc[row];
                if (src != nullptr) cp_async16(d, src + cell);  // padding rows only feed discarded outputs
            }
        } else {
            for (int row = row0; row < nrows; row += 4, d += 4 * kFfRow)
                *reinterpret_cast<float4 *>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        cp_async_commit();
    };

    const int gl = lane >> 2, hl = lane & 3;
    const int a_row = P.a_slot[0] + gl;  // rows a_row + 8 r
    const int b_row = P.b_slot[0] + hl;  // rows b_row + 4 q
    int gofs[RB];                        // staged G row of each window row (MG)
#pragma unroll
    for (int r = 0; r < RB; ++r) gofs[r] = (MG ? X.grow[gl + 8 * r] : P.g_row) * kFfRow;
    // FP32 partials are folded every kFfFold chunks into this warp's own FP64
    // partial in global memory (L2 resident), keeping registers for the tile
    double *dst = partial + ((int64_t)blockIdx.x * kFfWarps + warp) * (WR * WC);
    float2 acc[RB][CB];
#pragma unroll
    for (int r = 0; r < RB; ++r)
#pragma unroll
        for (int q = 0; q < CB; ++q) acc[r][q] = make_float2(0.f, 0.f);
    bool stored = false;
    auto fold = [&]() {
#pragma unroll
        for (int r = 0; r < RB; ++r)
#pragma unroll
            for (int q = 0; q < CB; ++q) {
                double *p = dst + (gl + 8 * r) * WC + hl + 4 * q;
                *p = (stored ? *p : 0.0) + ((double)acc[r][q].x + (double)acc[r][q].y);
                acc[r][q] = make_float2(0.f, 0.f);
            }
        stored = true;
    };
    // NBUF-deep ring per warp: chunks k+1 .. k+NBUF-1 stream in while chunk k
    // is contracted; an empty commit keeps one cp.async group per chunk slot
    for (int j = 0; j < NBUF - 1; ++j) {
        if (j < nchunk) issue(j, j);
        else cp_async_commit();
    }
    for (int k = 0; k < nchunk; ++k) {
        const int kn = k + NBUF - 1;
        if (kn < nchunk) issue(kn, kn % NBUF);
        else cp_async_commit();
        cp_async_wait<NBUF - 1>();  // the group of chunk k has landed
        __syncwarp();
        const float *sb = buf0 + (k % NBUF) * slab;
        const float *rg = sb + P.g_row * kFfRow;
        const float *ra = sb + a_row * kFfRow;
        const float *rb = sb + b_row * kFfRow;
#pragma unroll 4
        for (int c = 0; c < 32; c += 2) {
            const float2 g2 = *reinterpret_cast<const float2 *>(rg + c);
            float2 a2[RB], b2[CB];
#pragma unroll
            for (int r = 0; r < RB; ++r)
                a2[r] = __fmul2_rn(MG ? *reinterpret_cast<const float2 *>(sb + gofs[r] + c) : g2,
                                   *reinterpret_cast<const float2 *>(ra + 8 * r * kFfRow + c));
#pragma unroll
            for (int q = 0; q < CB; ++q) b2[q] = *reinterpret_cast<const float2 *>(rb + 4 * q * kFfRow + c);
#pragma unroll
            for (int r = 0; r < RB; ++r)
#pragma unroll
                for (int q = 0; q < CB; ++q) acc[r][q] = __ffma2_rn(a2[r], b2[q], acc[r][q]);
        }
        __syncwarp();  // this slot is refilled by the issue of iteration k + 1
        if ((k + 1) % kFfFold == 0) fold();
    }
    fold();  // also defines the partial of a warp that had no chunk
}

// out[i nb + j] = the sum over the parts p of partial[p][i][j], in a fixed
// order (bitwise reproducible): block b takes the 32 window entries
// e = 32 b + lane (e = i wc + j), warp w sums the parts w, w + 32, ... of its
// lane's entry (each warp load reads 32 consecutive entries of one part), and
// the 32 warp sums are added in warp order.
constexpr int kReduceWarps = 32;
__global__ void __launch_bounds__(32 * kReduceWarps)
    gram_window_reduce_kernel(const double *partial, int nparts, int wr, int wc, int na, int nb, double *out) {
    __shared__ double ws[kReduceWarps][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int e = blockIdx.x * 32 + lane;
    const int64_t W = (int64_t)wr * wc;
    double s = 0.0;
    if (e < na * wc) {
#pragma unroll 4
        for (int p = warp; p < nparts; p += kReduceWarps) s += partial[p * W + e];
    }
    ws[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && e < na * wc) {
        double t = 0.0;
        for (int w = 0; w < kReduceWarps; ++w) t += ws[w][lane];
        const int i = e / wc, j = e - (e / wc) * wc;
        if (j < nb) out[i * nb + j] = t;
    }
}

static inline void launch_window_reduce(const double *partial, int nparts, int wr, int wc, int na, int nb,
                                        double *out, cudaStream_t s) {
    gram_window_reduce_kernel<<<(na * wc + 31) / 32, 32 * kReduceWarps, 0, s>>>(partial, nparts, wr, wc, na, nb, out);
}

// Staged rows and window of an FP32 Gram launch (na <= 48, nb <= 24).
struct FfPlan {
    GramParams P;
    int RB, CB, wr, wc, nbuf;
    size_t smem;
};

static bool ff_plan(int64_t ncell, int64_t stride, const int *a, int na, const int *b, int nb, FfPlan *pl,
                    int ngs = 1) {
    GramParams &P = pl->P;
    std::memset(&P, 0, sizeof(P));
    pl->RB = (na + 7) / 8;
    pl->CB = (nb + 3) / 4;
    if (pl->RB > 6 || pl->CB > 6) return false;
    pl->wr = 8 * pl->RB;
    pl->wc = 4 * pl->CB;
    P.na = na;
    P.nb = nb;
    // staged rows: [G][A window][B window unless B is a contiguous run of A whose
    // window stays inside the A window]
    int b_off = -1;
    for (int off = 0; off + nb <= na && b_off < 0; ++off) {
        bool same = true;
        for (int j = 0; j < nb && same; ++j) same = a[off + j] == b[j];
        if (same && off + pl->wc <= pl->wr) b_off = off;
    }
    std::vector<int> rows;
    for (int j = 0; j < ngs; ++j) rows.push_back(-2 - j);  // weight fields G_j
    for (int i = 0; i < pl->wr; ++i) rows.push_back(i < na ? a[i] : -1);
    const int b_base = b_off >= 0 ? ngs + b_off : (int)rows.size();
    if (b_off < 0)
        for (int j = 0; j < pl->wc; ++j) rows.push_back(j < nb ? b[j] : -1);
    if ((int)rows.size() > kFfMaxRows) return false;
    P.nunion = (int)rows.size();
    for (int u = 0; u < P.nunion; ++u) P.union_field[u] = rows[u];
    P.g_row = 0;
    P.a_slot[0] = ngs;
    P.b_slot[0] = b_base;
    P.ncell = ncell;
    P.field_stride = stride;
    // two blocks per SM: ~110 KB of slabs each
    const size_t per_buf = (size_t)kFfWarps * P.nunion * kFfRow * sizeof(float);
    pl->nbuf = (int)std::min<size_t>(4, (110 * 1024 - kFfTable) / per_buf);
    pl->smem = kFfTable + pl->nbuf * per_buf;
    return pl->nbuf >= 2;
}

template <int R_, int C_, bool MG>
static cudaError_t ff_launch_rc(const FfPlan &pl, int nblocks, const float *g, const float *fields,
                                const FfMulti &X, double *part, cudaStream_t s) {
    cudaError_t e;
#define CNPC_FF_NB(NB_)                                                                                          \
    if (pl.nbuf == NB_) {                                                                                        \
        e = cudaFuncSetAttribute(gram_ffma_kernel<R_, C_, NB_, MG>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (int)pl.smem);                                                                  \
        if (e != cudaSuccess) return e;                                                                          \
        gram_ffma_kernel<R_, C_, NB_, MG><<<nblocks, kFfWarps * 32, pl.smem, s>>>(g, fields, pl.P, X, part);     \
        return cudaGetLastError();                                                                               \
    }
    CNPC_FF_NB(2) CNPC_FF_NB(3) CNPC_FF_NB(4)
#undef CNPC_FF_NB
    return cudaErrorInvalidValue;
}

template <bool MG>
static cudaError_t ff_launch(const FfPlan &pl, int nblocks, const float *g, const float *fields, const FfMulti &X,
                             double *part, cudaStream_t s) {
#define CNPC_FF_CASE(R_, C_) \
    if (pl.RB == R_ && pl.CB == C_) return ff_launch_rc<R_, C_, MG>(pl, nblocks, g, fields, X, part, s);
#define CNPC_FF_ROW(R_) \
    CNPC_FF_CASE(R_, 1) CNPC_FF_CASE(R_, 2) CNPC_FF_CASE(R_, 3) CNPC_FF_CASE(R_, 4) CNPC_FF_CASE(R_, 5) CNPC_FF_CASE(R_, 6)
    CNPC_FF_ROW(1) CNPC_FF_ROW(2) CNPC_FF_ROW(3) CNPC_FF_ROW(4) CNPC_FF_ROW(5) CNPC_FF_ROW(6)
#undef CNPC_FF_ROW
#undef CNPC_FF_CASE
    return cudaErrorInvalidValue;
}

static int run_gram_ffma(cnpc_ctx *ctx, int64_t ncell, const float *g, const float *fields, int64_t stride,
                         const int *a, int na, const int *b, int nb, double *out, cudaStream_t s) {
    CNPC_REQUIRE(ctx, ((stride * sizeof(float)) % 16 == 0) && (ncell % 4 == 0) && ((uintptr_t)g % 16 == 0) &&
                          ((uintptr_t)fields % 16 == 0),
                 "contraction needs 16-byte aligned fields, field_stride and ncell");
    FfPlan pl;
    CNPC_REQUIRE(ctx, ff_plan(ncell, stride, a, na, b, nb, &pl),
                 "FP32 Gram launch covers at most 48 x 24 outputs");
    const int64_t nchunks = (ncell + kFfChunk - 1) / kFfChunk;
    const int nblocks = (int)std::min<int64_t>(2 * ctx->num_sms, nchunks);
    const int nparts = nblocks * kFfWarps;
    int st = ensure_scratch(ctx, (size_t)nparts * pl.wr * pl.wc * sizeof(double) + 256, s);
    if (st) return st;
    double *part = (double *)ctx->scratch;
    FfMulti X;
    std::memset(&X, 0, sizeof(X));
    st = check_cuda(ctx, ff_launch<false>(pl, nblocks, g, fields, X, part, s), "gram_ffma_kernel");
    if (st) return st;
    launch_window_reduce(part, nparts, pl.wr, pl.wc, na, nb, out, s);
    return check_launch(ctx, "gram_window_reduce_kernel");
}

// Several weight fields in one FP32 launch: out[i, j] = sum_x G_{ag[i]} F_{a_i} F_{b_j}.
static int run_gram_ffma_mg(cnpc_ctx *ctx, int64_t ncell, const float *const *gs, int ngs, const float *fields,
                            int64_t stride, const int *a, const int *ag, int na, const int *b, int nb, double *out,
                            cudaStream_t s) {
    CNPC_REQUIRE(ctx, ((stride * sizeof(float)) % 16 == 0) && (ncell % 4 == 0) && ((uintptr_t)fields % 16 == 0),
                 "contraction needs 16-byte aligned fields, field_stride and ncell");
    FfPlan pl;
    CNPC_REQUIRE(ctx, ff_plan(ncell, stride, a, na, b, nb, &pl, ngs),
                 "FP32 multi-weight Gram launch covers at most 48 x 24 outputs");
    FfMulti X;
    std::memset(&X, 0, sizeof(X));
    for (int j = 0; j < ngs; ++j) {
        CNPC_REQUIRE(ctx, gs[j] != nullptr && (uintptr_t)gs[j] % 16 == 0, "weight fields must be 16-byte aligned");
        X.g[j] = gs[j];
    }
    for (int i = 0; i < na; ++i) X.grow[i] = ag[i];
    const int64_t nchunks = (ncell + kFfChunk - 1) / kFfChunk;
    const int nblocks = (int)std::min<int64_t>(2 * ctx->num_sms, nchunks);
    const int nparts = nblocks * kFfWarps;
    int st = ensure_scratch(ctx, (size_t)nparts * pl.wr * pl.wc * sizeof(double) + 256, s);
    if (st) return st;
    double *part = (double *)ctx->scratch;
    st = check_cuda(ctx, ff_launch<true>(pl, nblocks, gs[0], fields, X, part, s), "gram_ffma_kernel");
    if (st) return st;
    launch_window_reduce(part, nparts, pl.wr, pl.wc, na, nb, out, s);
    return check_launch(ctx, "gram_window_reduce_kernel");
}

// out[i, j] = sum over every block of the group owning tile(i, j) and every
// warp of that block assigned to the tile, in a fixed order.
template <int TM, int TN, int NW>
__global__ void gram_reduce_kernel(const double *partial, int nblocks, int ngroups, int ntiles, int ct,
                                   int na, int nb, double *out) {
    const int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= na * nb) return;
    const int i = o / nb, j = o % nb;
    const int tile = (i / TM) * ct + (j / TN);
    const int e = (i % TM) * TN + (j % TN);
    const int group = tile / NW;
    const int nt = min(NW, ntiles - group * NW);
    const int local = tile - group * NW;
    const int per_block = (NW - 1 - local) / nt + 1;  // warps of a block assigned to this tile
    const int nblk = (nblocks - group + ngroups - 1) / ngroups;
    double s = 0.0;
    for (int q = lane; q < nblk * per_block; q += 32) {
        const int b = group + (q / per_block) * ngroups;
        const int w = local + (q % per_block) * nt;
        s += partial[((int64_t)b * NW + w) * (TM * TN) + e];
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) out[o] = s;
}

template <typename T>
static int run_gram(cnpc_ctx *ctx, int64_t ncell, const T *g, const T *fields, int64_t stride,
                    const int *a, int na, const int *b, int nb, double *out, cudaStream_t s) {
    using Tile = typename TileOf<T>::type;
    constexpr int TM = Tile::TM, TN = Tile::TN, NW = Tile::WARPS, CHUNK = Tile::CHUNK;
    GramParams P;
    std::memset(&P, 0, sizeof(P));
    P.na = na;
    P.nb = nb;
    // staged rows: [G][A rows padded to TM][B rows padded to TN unless B is a
    // contiguous run of A], so each tile's rows are consecutive
    const int na_pad = (na + TM - 1) / TM * TM;
    const int nb_pad = (nb + TN - 1) / TN * TN;
    int b_off = -1;
    for (int off = 0; off + nb <= na && b_off < 0; ++off) {
        bool same = true;
        for (int j = 0; j < nb && same; ++j) same = a[off + j] == b[j];
        // the padded columns must also stay inside the staged rows
        if (same && off + nb_pad <= na_pad) b_off = off;
    }
    std::vector<int> rows;
    rows.push_back(-2);  // G
    for (int i = 0; i < na_pad; ++i) rows.push_back(i < na ? a[i] : -1);
    int b_base = b_off >= 0 ? 1 + b_off : (int)rows.size();
    if (b_off < 0)
        for (int j = 0; j < nb_pad; ++j) rows.push_back(j < nb ? b[j] : -1);
    CNPC_REQUIRE(ctx, (int)rows.size() <= kMaxUnion, "too many staged rows (max 256)");
    P.nunion = (int)rows.size();
    P.ncopy = 0;
    for (int u = 0; u < P.nunion; ++u) {
        P.union_field[u] = rows[u];
        if (rows[u] != -1) ++P.ncopy;
    }
    P.g_row = 0;
    for (int i = 0; i < na; ++i) P.a_slot[i] = 1 + i;
    for (int j = 0; j < nb; ++j) P.b_slot[j] = b_base + j;
    const int rtiles = na_pad / TM;
    P.ct = nb_pad / TN;
    P.ntiles = rtiles * P.ct;
    P.ngroups = (P.ntiles + NW - 1) / NW;
    P.ncell = ncell;
    P.field_stride = stride;
    CNPC_REQUIRE(ctx, ((stride * sizeof(T)) % 16 == 0) && ((ncell * sizeof(T)) % 16 == 0) &&
                          ((uintptr_t)g % 16 == 0) && ((uintptr_t)fields % 16 == 0),
                 "contraction needs 16-byte aligned fields, field_stride and ncell");
    const size_t row_bytes = (size_t)CHUNK * sizeof(T);
    P.nstages = (int)std::min<size_t>(kMaxStages, (220 * 1024) / (P.nunion * row_bytes));
    CNPC_REQUIRE(ctx, P.nstages >= 2, "too many staged rows for the shared-memory ring (max 110)");
    const size_t smem = (size_t)P.nstages * P.nunion * row_bytes;
    P.flush_chunks = 1 << 30;  // FP64 accumulators throughout
    P.wait_limit = ctx->wait_limit;
    int st = check_cuda(ctx, cudaFuncSetAttribute(gram_kernel<T, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem), "gram smem attribute");
    if (st) return st;
    st = ensure_status(ctx);
    if (st) return st;
    const int64_t nchunks = (ncell + CHUNK - 1) / CHUNK;
    int64_t nxr = std::min<int64_t>(std::max<int64_t>(1, ctx->num_sms / P.ngroups), nchunks);
    const int nblocks = (int)(nxr * P.ngroups);
    const size_t partial_bytes = (size_t)nblocks * NW * TM * TN * sizeof(double) + 256;
    st = ensure_scratch(ctx, partial_bytes, s);
    if (st) return st;
    // a wait that gives up sets the context's status word (sticky until
    // cnpc_ctx_take_status) and makes this call's outputs NaN
    gram_kernel<T, NW><<<(unsigned)nblocks, NW * 32, smem, s>>>(g, fields, P, (double *)ctx->scratch,
                                                                 ctx->d_status);
    st = check_launch(ctx, "gram_kernel");
    if (st) return st;
    const int nout = na * nb;
    gram_reduce_kernel<TM, TN, NW><<<(nout + 7) / 8, 256, 0, s>>>(
        (const double *)ctx->scratch, nblocks, P.ngroups, P.ntiles, P.ct, na, nb, out);
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
        return run_gram_ffma(ctx, ncell, (const float *)d_g, (const float *)d_fields, field_stride, h_a, na,
                             h_b, nb, d_out, s);
    return run_gram<double>(ctx, ncell, (const double *)d_g, (const double *)d_fields, field_stride,
                            h_a, na, h_b, nb, d_out, s);
}

int cnpc_contract_gram_multi_g(cnpc_ctx *ctx, int64_t ncell, const float *const *h_gs, int ngs,
                               const float *d_fields, int64_t field_stride, const int *h_a, const int *h_ag,
                               int na, const int *h_b, int nb, double *d_out, cnpc_stream_t stream) {
    int st = check_contract(ctx, CNPC_F32, ncell, h_gs ? h_gs[0] : nullptr, d_fields, field_stride);
    if (st) return st;
    CNPC_REQUIRE(ctx, h_a && h_ag && h_b && d_out, "null argument");
    CNPC_REQUIRE(ctx, ngs >= 1 && ngs <= 4, "ngs must be 1..4");
    CNPC_REQUIRE(ctx, na >= 1 && na <= 48 && nb >= 1 && nb <= 24, "multi-weight Gram covers 1..48 x 1..24 outputs");
    for (int i = 0; i < na; ++i) {
        CNPC_REQUIRE(ctx, h_a[i] >= 0, "negative field index");
        CNPC_REQUIRE(ctx, h_ag[i] >= 0 && h_ag[i] < ngs, "row weight index out of range");
    }
    for (int j = 0; j < nb; ++j) CNPC_REQUIRE(ctx, h_b[j] >= 0, "negative field index");
    return run_gram_ffma_mg(ctx, ncell, h_gs, ngs, d_fields, field_stride, h_a, h_ag, na, h_b, nb, d_out,
                            (cudaStream_t)stream);
}

}  // extern "C"

// ===========================================================================
// Allocation-free variant of cnpc_contract_gram.
//
// Some callers cannot let a library call cudaMalloc: an application that
// hands the whole device to its own memory pool up front (so a library
// allocation would fail or fragment the pool), or a pipeline that keeps other
// streams busy and cannot afford the device-wide synchronisation that
// cudaFree (and a growing cudaMalloc) may impose.  For them the per-block
// partial sums of the contraction live in one fixed array in the library's
// device memory instead of the context's scratch buffer.
// ===========================================================================
namespace cnpc {

// 8 MiB of doubles per device: per-block partials plus a status word.  Every
// GPU that loads the library holds this array until the process exits.
constexpr size_t kNoAllocDoubles = (size_t)1 << 20;
constexpr size_t kNoAllocStatusSlot = kNoAllocDoubles - 32;  // last 256 bytes
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[kNoAllocMaxDevices];
static int g_noalloc_sms[kNoAllocMaxDevices];

// Device address of the array for the current device.  The symbol's name in
// host code is only a stand-in, so the address is fetched with
// cudaGetSymbolAddress once per device (with that device current) and cached.
static int noalloc_scratch(double **ptr, int *sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CNPC_ECUDA;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return CNPC_EINVAL;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return CNPC_ECUDA;
        }
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            return CNPC_ECUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double *>(p);
        g_noalloc_sms[dev] = n;
    }
    *ptr = g_noalloc_ptr[dev];
    *sms = g_noalloc_sms[dev];
    return CNPC_OK;
}

static int noalloc_cuda(cudaError_t e) {
    if (e == cudaSuccess) return CNPC_OK;
    cudaGetLastError();
    return CNPC_ECUDA;
}

static int noalloc_gram_f32(int64_t ncell, const float *g, const float *fields, int64_t stride, const int *a,
                            int na, const int *b, int nb, double *out, cudaStream_t s) {
    if (((stride * sizeof(float)) % 16) || (ncell % 4) || ((uintptr_t)g % 16) || ((uintptr_t)fields % 16))
        return CNPC_EINVAL;
    FfPlan pl;
    if (!ff_plan(ncell, stride, a, na, b, nb, &pl)) return CNPC_EINVAL;  // one launch: at most 48 x 24
    double *scratch = nullptr;
    int sms = 0;
    int st = noalloc_scratch(&scratch, &sms);
    if (st) return st;
    // as many blocks as the fixed array can hold partials for
    const size_t per_block = (size_t)kFfWarps * pl.wr * pl.wc;
    const int64_t nchunks = (ncell + kFfChunk - 1) / kFfChunk;
    const int nblocks =
        (int)std::min<int64_t>(std::min<int64_t>(2 * sms, nchunks), kNoAllocStatusSlot / per_block);
    if (nblocks < 1) return CNPC_EINVAL;
    FfMulti X;
    std::memset(&X, 0, sizeof(X));
    st = noalloc_cuda(ff_launch<false>(pl, nblocks, g, fields, X, scratch, s));
    if (st) return st;
    launch_window_reduce(scratch, nblocks * kFfWarps, pl.wr, pl.wc, na, nb, out, s);
    return noalloc_cuda(cudaGetLastError());
}

static int noalloc_gram_f64(int64_t ncell, const double *g, const double *fields, int64_t stride, const int *a,
                            int na, const int *b, int nb, double *out, cudaStream_t s) {
    using Tile = Fp64Tile;
    constexpr int TM = Tile::TM, TN = Tile::TN, NW = Tile::WARPS, CHUNK = Tile::CHUNK;
    if (((stride * sizeof(double)) % 16) || ((ncell * sizeof(double)) % 16) || ((uintptr_t)g % 16) ||
        ((uintptr_t)fields % 16))
        return CNPC_EINVAL;
    double *scratch = nullptr;
    int sms = 0;
    int st = noalloc_scratch(&scratch, &sms);
    if (st) return st;
    GramParams P;
    std::memset(&P, 0, sizeof(P));
    P.na = na;
    P.nb = nb;
    const int na_pad = (na + TM - 1) / TM * TM;
    const int nb_pad = (nb + TN - 1) / TN * TN;
    int b_off = -1;
    for (int off = 0; off + nb <= na && b_off < 0; ++off) {
        bool same = true;
        for (int j = 0; j < nb && same; ++j) same = a[off + j] == b[j];
        if (same && off + nb_pad <= na_pad) b_off = off;
    }
    std::vector<int> rows;
    rows.push_back(-2);
    for (int i = 0; i < na_pad; ++i) rows.push_back(i < na ? a[i] : -1);
    const int b_base = b_off >= 0 ? 1 + b_off : (int)rows.size();
    if (b_off < 0)
        for (int j = 0; j < nb_pad; ++j) rows.push_back(j < nb ? b[j] : -1);
    if ((int)rows.size() > kMaxUnion) return CNPC_EINVAL;
    P.nunion = (int)rows.size();
    for (int u = 0; u < P.nunion; ++u) {
        P.union_field[u] = rows[u];
        if (rows[u] != -1) ++P.ncopy;
    }
    P.g_row = 0;
    for (int i = 0; i < na; ++i) P.a_slot[i] = 1 + i;
    for (int j = 0; j < nb; ++j) P.b_slot[j] = b_base + j;
    P.ct = nb_pad / TN;
    P.ntiles = (na_pad / TM) * P.ct;
    P.ngroups = (P.ntiles + NW - 1) / NW;
    P.ncell = ncell;
    P.field_stride = stride;
    const size_t row_bytes = (size_t)CHUNK * sizeof(double);
    P.nstages = (int)std::min<size_t>(kMaxStages, (220 * 1024) / (P.nunion * row_bytes));
    if (P.nstages < 2) return CNPC_EINVAL;
    const size_t smem = (size_t)P.nstages * P.nunion * row_bytes;
    P.flush_chunks = 1 << 30;
    P.wait_limit = kWaitLimit;
    const size_t per_block = (size_t)NW * TM * TN;
    const int64_t nchunks = (ncell + CHUNK - 1) / CHUNK;
    int64_t nxr = std::min<int64_t>(std::max<int64_t>(1, sms / P.ngroups), nchunks);
    nxr = std::min<int64_t>(nxr, (int64_t)(kNoAllocStatusSlot / per_block) / P.ngroups);
    if (nxr < 1) return CNPC_EINVAL;
    const int nblocks = (int)(nxr * P.ngroups);
    int *status = reinterpret_cast<int *>(scratch + kNoAllocStatusSlot);
    // the shared array keeps the previous call's contents: the bounded-wait
    // status word must start at zero
    st = noalloc_cuda(cudaMemsetAsync(status, 0, sizeof(int), s));
    if (st) return st;
    st = noalloc_cuda(
        cudaFuncSetAttribute(gram_kernel<double, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (st) return st;
    gram_kernel<double, NW><<<(unsigned)nblocks, NW * 32, smem, s>>>(g, fields, P, scratch, status);
    st = noalloc_cuda(cudaGetLastError());
    if (st) return st;
    const int nout = na * nb;
    gram_reduce_kernel<TM, TN, NW><<<(nout + 7) / 8, 256, 0, s>>>(scratch, nblocks, P.ngroups, P.ntiles, P.ct, na,
                                                                  nb, out);
    return noalloc_cuda(cudaGetLastError());
}

}  // namespace cnpc

extern "C" int cnpc_contract_gram_noalloc(int dtype, int64_t ncell, const void *d_g, const void *d_fields,
                                          int64_t field_stride, const int *h_a, int na, const int *h_b, int nb,
                                          double *d_out, cnpc_stream_t stream) {
    if (dtype != CNPC_F32 && dtype != CNPC_F64) return CNPC_EINVAL;
    if (ncell < 1 || !d_g || !d_fields || !h_a || !h_b || !d_out || field_stride < ncell) return CNPC_EINVAL;
    if (na < 1 || na > kMaxRows || nb < 1 || nb > kMaxRows) return CNPC_EINVAL;
    for (int i = 0; i < na; ++i)
        if (h_a[i] < 0) return CNPC_EINVAL;
    for (int j = 0; j < nb; ++j)
        if (h_b[j] < 0) return CNPC_EINVAL;
    try {
        cudaStream_t s = (cudaStream_t)stream;
        if (dtype == CNPC_F32)
            return noalloc_gram_f32(ncell, (const float *)d_g, (const float *)d_fields, field_stride, h_a, na, h_b,
                                    nb, d_out, s);
        return noalloc_gram_f64(ncell, (const double *)d_g, (const double *)d_fields, field_stride, h_a, na, h_b,
                                nb, d_out, s);
    } catch (...) {
        return CNPC_EINVAL;
    }
}
