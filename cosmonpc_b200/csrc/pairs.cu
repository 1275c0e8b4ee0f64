// Pair-list contraction: out[p] = sum_x G(x) F_{a_p}(x) F_{b_p}(x) for a list of
// (a_p, b_p) field pairs.  The diagonal data vector of the bispectrum
// (clustering_estimator.py:1983-2035 survey, ce:998-1061 box) needs only the
// same-bin pairs, a few per bin, where the Gram form would compute the whole
// bins x bins block; this streams G and every listed field once per chunk of
// pairs, four cells per thread per step, FP32 products folded into FP64 every
// 64 cells (FP64 throughout for FP64 fields), per-block partials reduced in a
// fixed order.
#include <cstring>

#include "internal.h"

namespace cnpc {

constexpr int kPairChunk = 8;      // pairs per pass over the cells
constexpr int kPairThreads = 256;
constexpr int kPairMax = 256;

struct PairList {
    int n;
    int a[kPairMax];
    int b[kPairMax];
};

template <typename T> struct Vec4;
template <> struct Vec4<float> {
    using type = float4;
};
template <> struct Vec4<double> {
    using type = double4;
};

template <typename T>
__global__ void __launch_bounds__(kPairThreads) pair_sums_kernel(const T *__restrict__ g, const T *__restrict__ f,
                                                                 int64_t stride, int64_t nvec, PairList pl, int p0,
                                                                 int np, double *partial) {
    using V = typename Vec4<T>::type;
    const V *g4 = reinterpret_cast<const V *>(g);
    const V *fa[kPairChunk], *fb[kPairChunk];
#pragma unroll
    for (int q = 0; q < kPairChunk; ++q) {
        const int p = p0 + (q < np ? q : 0);
        fa[q] = reinterpret_cast<const V *>(f + (int64_t)pl.a[p] * stride);
        fb[q] = reinterpret_cast<const V *>(f + (int64_t)pl.b[p] * stride);
    }
    double acc[kPairChunk];
    T part[kPairChunk];
#pragma unroll
    for (int q = 0; q < kPairChunk; ++q) acc[q] = 0.0, part[q] = (T)0;
    int since = 0;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvec; v += step) {
        const V gv = g4[v];
#pragma unroll
        for (int q = 0; q < kPairChunk; ++q) {
            if (q < np) {
                const V x = fa[q][v], y = fb[q][v];
                part[q] += gv.x * x.x * y.x + gv.y * x.y * y.y + gv.z * x.z * y.z + gv.w * x.w * y.w;
            }
        }
        if (++since == 16) {  // 64 cells per thread in FP32, then into the FP64 sum
#pragma unroll
            for (int q = 0; q < kPairChunk; ++q) acc[q] += (double)part[q], part[q] = (T)0;
            since = 0;
        }
    }
    __shared__ double red[kPairThreads / 32][kPairChunk];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kPairChunk; ++q) {
        double s = acc[q] + (double)part[q];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][q] = s;
    }
    __syncthreads();
    if (threadIdx.x < np) {
        double s = 0.0;
        for (int w = 0; w < kPairThreads / 32; ++w) s += red[w][threadIdx.x];
        partial[(int64_t)blockIdx.x * kPairMax + p0 + threadIdx.x] = s;
    }
}

// out[p] = sum over blocks of partial[block][p] (one warp per output, fixed order)
__global__ void pair_reduce_kernel(const double *partial, int nblocks, int npairs, double *out) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= npairs) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partial[(int64_t)b * kPairMax + p];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[p] = s;
}

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_contract_pairs(cnpc_ctx *ctx, int dtype, int64_t ncell, const void *d_g, const void *d_fields,
                                   int64_t field_stride, const int *h_a, const int *h_b, int npairs, double *d_out,
                                   cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    CNPC_REQUIRE(ctx, d_g && d_fields && d_out && h_a && h_b, "null argument");
    CNPC_REQUIRE(ctx, npairs >= 1 && npairs <= kPairMax, "npairs out of range (1..256)");
    CNPC_REQUIRE(ctx, ncell > 0 && ncell % 4 == 0, "ncell must be a positive multiple of 4");
    CNPC_REQUIRE(ctx, field_stride >= ncell && field_stride % 4 == 0, "field_stride must be >= ncell, multiple of 4");
    const size_t esz = dtype == CNPC_F32 ? sizeof(float) : sizeof(double);
    const size_t align = 4 * esz;
    CNPC_REQUIRE(ctx, reinterpret_cast<uintptr_t>(d_g) % align == 0 && reinterpret_cast<uintptr_t>(d_fields) % align == 0,
                 "G and fields must be aligned to 4 elements");
    PairList pl;
    pl.n = npairs;
    for (int p = 0; p < npairs; ++p) {
        CNPC_REQUIRE(ctx, h_a[p] >= 0 && h_b[p] >= 0, "negative field index");
        pl.a[p] = h_a[p];
        pl.b[p] = h_b[p];
    }
    const int64_t nvec = ncell / 4;
    int64_t want = (nvec + kPairThreads - 1) / kPairThreads;
    const int nblocks = (int)(want < (int64_t)ctx->num_sms * 4 ? (want > 0 ? want : 1) : (int64_t)ctx->num_sms * 4);
    cudaStream_t s = (cudaStream_t)stream;
    int st = ensure_scratch(ctx, sizeof(double) * (size_t)nblocks * kPairMax, s);
    if (st) return st;
    double *partial = static_cast<double *>(ctx->scratch);
    for (int p0 = 0; p0 < npairs; p0 += kPairChunk) {
        const int np = npairs - p0 < kPairChunk ? npairs - p0 : kPairChunk;
        if (dtype == CNPC_F32)
            pair_sums_kernel<float><<<nblocks, kPairThreads, 0, s>>>((const float *)d_g, (const float *)d_fields,
                                                                     field_stride, nvec, pl, p0, np, partial);
        else
            pair_sums_kernel<double><<<nblocks, kPairThreads, 0, s>>>((const double *)d_g, (const double *)d_fields,
                                                                      field_stride, nvec, pl, p0, np, partial);
    }
    pair_reduce_kernel<<<(npairs * 32 + 255) / 256, 256, 0, s>>>(partial, nblocks, npairs, d_out);
    return check_launch(ctx, "pair_sums_kernel");
}
