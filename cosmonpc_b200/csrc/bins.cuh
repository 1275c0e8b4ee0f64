// Shared pieces of the k-space kernels: edge / harmonic tables passed by
// value, launch sizing, the warp-aggregated bin accumulator and argument checks.
#pragma once
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
