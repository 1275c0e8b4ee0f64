// Shared pieces of the k-space kernels: edge / harmonic tables passed by
// value, launch sizing, the warp-aggregated bin accumulator and argument checks.
#pragma once
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "internal.h"

namespace cnpc {

struct EdgeSet {
    int n;
    double e[CNPC_MAX_EDGES];
};
struct HarmTable {
    int n;
    cnpc_harmonic h[CNPC_MAX_HARMONICS];
};
struct ItemTable {
    int n;
    cnpc_shell_item it[CNPC_MAX_ITEMS];
};

inline int grid_for(cnpc_ctx *ctx, int64_t work, int threads, int per_sm = 8) {
    int64_t want = (work + threads - 1) / threads;
    int64_t cap = (int64_t)ctx->num_sms * per_sm;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

// Copy the edges to shared memory (a __syncthreads() follows before use):
// find_bin indexes them at run time, which on a by-value kernel parameter is a
// constant-bank load through the slow address-divergence path for every probe.
__device__ inline double *edges_to_shared(double *s, const EdgeSet &es) {
    for (int i = threadIdx.x; i < es.n; i += blockDim.x) s[i] = es.e[i];
    return s;
}

// Sum v into bins s[bin] over the lanes of a warp (all 32 lanes must call;
// bin < 0 means "no contribution").
__device__ inline void warp_bin_add(double *s, int bin, double v) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned active = __ballot_sync(full, bin >= 0);
    while (active) {
        const int leader = __ffs(active) - 1;
        const int b = __shfl_sync(full, bin, leader);
        const unsigned same = __ballot_sync(full, bin == b);
        double x = (bin == b) ? v : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(full, x, o);
        if (lane == leader) atomicAdd(&s[b], x);
        active &= ~same;
    }
}

// Sum V values per bin over the lanes of a warp, value i of bin b into
// s[b + i * stride] (all 32 lanes must call; bin < 0 means "no contribution").
// Consecutive modes along n_z meet the bins in increasing order, so equal bins
// sit in runs of adjacent lanes: a segmented inclusive scan sums each run and
// the run's last lane adds it, at a cost that does not grow with the number of
// bins a warp meets.  Any bin pattern gives the right sums (a bin split over
// several runs is added once per run).
template <int V>
__device__ inline void warp_run_add(double *s, int stride, int bin, double (&v)[V], int nv = V) {
    const unsigned full = 0xffffffffu;
    if (__ballot_sync(full, bin >= 0) == 0) return;
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(full, bin, 1);
    const unsigned heads = __ballot_sync(full, lane == 0 || prev != bin);
    // first lane of this lane's run: the highest head at or below it (bit 0 is a head)
    const int start = 31 - __clz(heads & (full >> (31 - lane)));
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const bool take = lane - o >= start;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            if (i >= nv) break;
            const double y = __shfl_up_sync(full, v[i], o);
            if (take) v[i] += y;
        }
    }
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
    if (tail && bin >= 0)
#pragma unroll
        for (int i = 0; i < V; ++i)
            if (i < nv) atomicAdd(&s[bin + i * stride], v[i]);
}

// Modes of the half spectrum with every |n_d| <= R (R < n/2): a compact index
// u over n_x, n_y in [-R, R], n_z in [0, R].  Shell sums only see modes below
// their last edge, so they iterate over that cube (R = -1: every mode).
struct BandIter {
    int n, R;
    int64_t count;
    __device__ __forceinline__ Mode mode(int64_t u, int64_t *t) const {
        if (R < 0) {
            *t = u;
            return mode_of(u, n);
        }
        const int w = 2 * R + 1, nzc = R + 1;
        int iz, jy, jx;
        if (u < ((int64_t)1 << 31)) {
            uint32_t rz, ry;
            const uint32_t r = udiv31((uint32_t)u, (uint32_t)nzc, &rz);
            jx = (int)udiv31(r, (uint32_t)w, &ry);
            iz = (int)rz;
            jy = (int)ry;
        } else {
            iz = (int)(u % nzc);
            const int64_t r = u / nzc;
            jy = (int)(r % w);
            jx = (int)(r / w);
        }
        Mode m;
        m.nx = jx - R;
        m.ny = jy - R;
        m.nz = iz;
        const int ix = m.nx < 0 ? m.nx + n : m.nx, iy = m.ny < 0 ? m.ny + n : m.ny;
        *t = ((int64_t)ix * n + iy) * (n / 2 + 1) + iz;
        m.mult = (iz == 0 || 2 * iz == n) ? 1 : 2;
        return m;
    }
};

inline BandIter band_iter(int n, double boxsize, double e_last) {
    BandIter b;
    b.n = n;
    const double kf = 2.0 * kPi / boxsize;
    const double r = e_last / kf * (1.0 + 1e-9);
    b.R = (r < 0.5 * n - 1.0) ? (int)std::floor(r) + 1 : -1;
    if (b.R >= 0 && 2 * b.R + 1 >= n) b.R = -1;
    b.count = b.R < 0 ? (int64_t)n * n * (n / 2 + 1) : (int64_t)(2 * b.R + 1) * (2 * b.R + 1) * (b.R + 1);
    return b;
}

inline int load_edges(cnpc_ctx *ctx, const double *h_edges, int nedges, EdgeSet *es) {
    CNPC_REQUIRE(ctx, h_edges != nullptr, "null edges");
    CNPC_REQUIRE(ctx, nedges >= 2 && nedges <= CNPC_MAX_EDGES, "nedges out of range (2..257)");
    for (int i = 0; i + 1 < nedges; ++i)
        CNPC_REQUIRE(ctx, h_edges[i] < h_edges[i + 1], "edges must be increasing");
    es->n = nedges;
    std::memcpy(es->e, h_edges, sizeof(double) * nedges);
    return CNPC_OK;
}

inline int check_common(cnpc_ctx *ctx, int dtype, int n, double boxsize) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    CNPC_REQUIRE(ctx, n >= 2 && n % 2 == 0 && n <= 2048, "n must be even, 2..2048");
    CNPC_REQUIRE(ctx, boxsize > 0.0, "boxsize must be positive");
    return CNPC_OK;
}

inline int64_t half_modes(int n) { return (int64_t)n * n * (n / 2 + 1); }

}  // namespace cnpc
