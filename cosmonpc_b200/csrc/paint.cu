// Mass assignment (pmesh ParticleMesh.paint restated): B-spline windows of
// order p = 1..4 on nodes at integer grid coordinates, periodic wrap; the
// interlaced +1/2-cell mesh is painted in the same pass.
#include <cmath>

#include "common.cuh"
#include "internal.h"

namespace cnpc {

// B-spline window W_p(s), s in grid units.
template <int P> __device__ inline double bspline(double s) {
    double a = fabs(s);
    if (P == 1) return a < 0.5 ? 1.0 : 0.0;
    if (P == 2) return a < 1.0 ? 1.0 - a : 0.0;
    if (P == 3) return a < 0.5 ? 0.75 - a * a : (a < 1.5 ? 0.5 * (1.5 - a) * (1.5 - a) : 0.0);
    // P == 4
    if (a < 1.0) return (4.0 - 6.0 * a * a + 3.0 * a * a * a) / 6.0;
    if (a < 2.0) return (2.0 - a) * (2.0 - a) * (2.0 - a) / 6.0;
    return 0.0;
}

template <int P> __device__ inline void axis_weights(double g, int n, int *idx, double *w) {
    int base = (P % 2 == 0) ? (int)floor(g) - (P / 2 - 1) : (int)floor(__dadd_rn(g, 0.5)) - (P - 1) / 2;
#pragma unroll
    for (int o = 0; o < P; ++o) {
        int node = base + o;
        w[o] = bspline<P>(__dsub_rn((double)node, g));
        int r = node % n;
        idx[o] = r < 0 ? r + n : r;
    }
}

template <typename T, int P>
__device__ inline void deposit(T *mesh, int n, double gx, double gy, double gz, double mass) {
    int ix[P], iy[P], iz[P];
    double wx[P], wy[P], wz[P];
    axis_weights<P>(gx, n, ix, wx);
    axis_weights<P>(gy, n, iy, wy);
    axis_weights<P>(gz, n, iz, wz);
#pragma unroll
    for (int a = 0; a < P; ++a) {
#pragma unroll
        for (int b = 0; b < P; ++b) {
            const double wab = mass * wx[a] * wy[b];
            const size_t row = ((size_t)ix[a] * n + iy[b]) * n;
#pragma unroll
            for (int c = 0; c < P; ++c) atomicAdd(mesh + row + iz[c], (T)(wab * wz[c]));
        }
    }
}

template <typename T, int P>
__global__ void paint_kernel(const double *__restrict__ pos, const double *__restrict__ weight,
                             int64_t np, int n, double scale, T *mesh, T *mesh_shifted) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        // separately rounded products and sums (no FMA contraction), so grid
        // coordinates match the restated pmesh affine transform bit for bit
        const double gx = __dmul_rn(pos[3 * i + 0], scale);
        const double gy = __dmul_rn(pos[3 * i + 1], scale);
        const double gz = __dmul_rn(pos[3 * i + 2], scale);
        const double mass = weight ? weight[i] : 1.0;
        deposit<T, P>(mesh, n, gx, gy, gz, mass);
        if (mesh_shifted)
            deposit<T, P>(mesh_shifted, n, __dadd_rn(gx, 0.5), __dadd_rn(gy, 0.5), __dadd_rn(gz, 0.5), mass);
    }
}

template <typename T>
static int launch_paint(cnpc_ctx *ctx, const double *pos, const double *w, int64_t np, int n,
                        double scale, int window, T *m1, T *m2, cudaStream_t s) {
    const int threads = 256;
    int64_t want = (np + threads - 1) / threads;
    int64_t cap = (int64_t)ctx->num_sms * 16;
    int blocks = (int)(want < cap ? (want > 0 ? want : 1) : cap);
    switch (window) {
        case 1: paint_kernel<T, 1><<<blocks, threads, 0, s>>>(pos, w, np, n, scale, m1, m2); break;
        case 2: paint_kernel<T, 2><<<blocks, threads, 0, s>>>(pos, w, np, n, scale, m1, m2); break;
        case 3: paint_kernel<T, 3><<<blocks, threads, 0, s>>>(pos, w, np, n, scale, m1, m2); break;
        case 4: paint_kernel<T, 4><<<blocks, threads, 0, s>>>(pos, w, np, n, scale, m1, m2); break;
        default: return fail(ctx, CNPC_EINVAL, "window must be 1..4");
    }
    return check_launch(ctx, "paint_kernel");
}

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_paint(cnpc_ctx *ctx, int dtype, const double *d_pos, const double *d_weight,
                          int64_t np, int n, double boxsize, int window, void *d_mesh,
                          void *d_mesh_shifted, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, n >= 2 && n <= 2048, "n out of range");
    CNPC_REQUIRE(ctx, boxsize > 0.0, "boxsize must be positive");
    CNPC_REQUIRE(ctx, np >= 0, "negative particle count");
    CNPC_REQUIRE(ctx, window >= 1 && window <= 4, "window must be 1..4");
    CNPC_REQUIRE(ctx, d_mesh != nullptr, "null mesh");
    CNPC_REQUIRE(ctx, np == 0 || d_pos != nullptr, "null positions");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t cells = (size_t)n * n * n;
    const size_t esz = dtype == CNPC_F32 ? sizeof(float) : sizeof(double);
    int st = check_cuda(ctx, cudaMemsetAsync(d_mesh, 0, cells * esz, s), "memset mesh");
    if (st) return st;
    if (d_mesh_shifted) {
        st = check_cuda(ctx, cudaMemsetAsync(d_mesh_shifted, 0, cells * esz, s), "memset mesh");
        if (st) return st;
    }
    if (np == 0) return CNPC_OK;
    const double scale = (double)n / boxsize;
    if (dtype == CNPC_F32)
        return launch_paint<float>(ctx, d_pos, d_weight, np, n, scale, window, (float *)d_mesh,
                                   (float *)d_mesh_shifted, s);
    return launch_paint<double>(ctx, d_pos, d_weight, np, n, scale, window, (double *)d_mesh,
                                (double *)d_mesh_shifted, s);
}
