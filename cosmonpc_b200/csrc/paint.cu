// Mass assignment (pmesh ParticleMesh.paint restated): B-spline windows of
// order p = 1..4 on nodes at integer grid coordinates, periodic wrap; the
// interlaced +1/2-cell mesh is painted in the same pass.
#include <algorithm>
#include <cmath>
#include <type_traits>

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

// Painting frame: grid coordinate g = (x - origin) * scale with each
// operation rounded separately (no FMA contraction), so grid coordinates match
// Position - boxcenter (mesh_generator.py:182-183) followed by the restated
// pmesh affine transform bit for bit; x - 0 is exact, so a zero origin is the
// plain transform.  Masses are weight * mass_scale.
struct Frame {
    double ox, oy, oz;
    double scale;
    double mass_scale;
};

__device__ inline void grid_coords(const double *pos, int64_t i, const Frame &f, double *g) {
    g[0] = __dmul_rn(__dsub_rn(pos[3 * i + 0], f.ox), f.scale);
    g[1] = __dmul_rn(__dsub_rn(pos[3 * i + 1], f.oy), f.scale);
    g[2] = __dmul_rn(__dsub_rn(pos[3 * i + 2], f.oz), f.scale);
}

__device__ inline double mass_of(const double *weight, int64_t i, const Frame &f) {
    return weight ? __dmul_rn(weight[i], f.mass_scale) : f.mass_scale;
}

template <typename T, int P>
__global__ void paint_kernel(const double *__restrict__ pos, const double *__restrict__ weight,
                             int64_t np, int n, Frame f, T *mesh, T *mesh_shifted) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        double g[3];
        grid_coords(pos, i, f, g);
        const double gx = g[0], gy = g[1], gz = g[2];
        const double mass = mass_of(weight, i, f);
        deposit<T, P>(mesh, n, gx, gy, gz, mass);
        if (mesh_shifted)
            deposit<T, P>(mesh_shifted, n, __dadd_rn(gx, 0.5), __dadd_rn(gy, 0.5), __dadd_rn(gz, 0.5), mass);
    }
}

template <typename T>
static int launch_paint(cnpc_ctx *ctx, const double *pos, const double *w, int64_t np, int n,
                        const Frame &scale, int window, T *m1, T *m2, cudaStream_t s) {
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

// ------------------------------------------------------------ tiled paint
// Particles are counting-sorted by the 16^3-cell tile of their base node
// floor(g); a block then deposits one tile's particles into a (16+4)^3
// shared-memory region per mesh (every node a particle of the tile can reach,
// for both the plain and the +1/2-shifted grid and every window order) and
// adds the region to the mesh with one global atomic per node.  Node
// selection and weights are those of the per-particle kernel.
//
// The region accumulates in 32-bit fixed point (integer shared atomics run
// about twice as fast as FP32 ones and make the sum order-independent).  The
// tile's scale 2^e is the finest one that cannot overflow: a node receives at
// most one deposit from each particle whose first stencil node lies in the
// (P+1) x (P+1) column window behind it (P+1 covers the shifted grid), so
// |sum| <= (max window count) x max|mass| x wmax^3 with wmax the largest 1-D
// weight of the window (e <= 100).  One particle's deposit is then resolved to
// (max window count) x 2^-31 of itself, while sums are exact; a tile whose
// window count exceeds 65536 (coarser than 2^-15 of one deposit) accumulates in
// FP32 instead.
constexpr int kTile = 16;
constexpr int kRegion = kTile + 4;  // nodes [b - 1, b + 3] of a base node b in the tile
constexpr int kRegionCells = kRegion * kRegion * kRegion;

__device__ inline int wrapi(int64_t v, int n) {
    // nodes are within one box length of [0, n) almost always: no 64-bit division
    if (v >= 0 && v < n) return (int)v;
    if (v < 0 && v >= -(int64_t)n) return (int)v + n;
    if (v >= n && v < 2 * (int64_t)n) return (int)(v - n);
    int r = (int)(v % n);
    return r < 0 ? r + n : r;
}

__global__ void tile_count_kernel(const double *__restrict__ pos, int64_t np, int n, Frame scale, int tpa,
                                  int *count, int *tile_of) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        double g[3];
        grid_coords(pos, i, scale, g);
        int tid = 0;
        for (int d = 0; d < 3; ++d) tid = tid * tpa + wrapi((int64_t)floor(g[d]), n) / kTile;
        tile_of[i] = tid;
        // clustered catalogs put many lanes of a warp in one tile: one atomic per tile
        const unsigned same = __match_any_sync(__activemask(), tid);
        if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&count[tid], __popc(same));
    }
}

// exclusive scan of count[0..nt) into offset[0..nt] and cursor (one block)
__global__ void tile_scan_kernel(const int *count, int nt, int *offset, int *cursor) {
    __shared__ long long part[1024];
    const int per = (nt + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(nt, b + per);
    long long s = 0;
    for (int i = b; i < e; ++i) s += count[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long run = 0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            const long long v = part[i];
            part[i] = run;
            run += v;
        }
    }
    __syncthreads();
    long long run = part[threadIdx.x];
    for (int i = b; i < e; ++i) {
        offset[i] = (int)run;
        cursor[i] = (int)run;
        run += count[i];
    }
    if (e == nt && b < e) offset[nt] = (int)run;
    if (nt == 0 && threadIdx.x == 0) offset[0] = 0;
}

__global__ void tile_scatter_kernel(const double *__restrict__ pos, const double *__restrict__ weight,
                                    int64_t np, Frame scale, const int *tile_of, int *cursor, double4 *sorted) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        double g[3];
        grid_coords(pos, i, scale, g);
        const int tid = tile_of[i];
        // reserve the slots of every lane in the same tile with one atomic
        const unsigned same = __match_any_sync(__activemask(), tid);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(same) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&cursor[tid], __popc(same));
        base = __shfl_sync(same, base, leader);
        const int slot = base + __popc(same & ((1u << lane) - 1));
        sorted[slot] = make_double4(g[0], g[1], g[2], mass_of(weight, i, scale));
    }
}

// no memory clobber: the region is only read after a __syncthreads
__device__ inline void red_shared_add_nc(int *addr, int v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(addr)), "r"(v));
}
__device__ inline void red_shared_add_nc(float *addr, float v) {
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(addr)), "f"(v));
}

// Region accumulator: fixed point (scale 2^e) or, for a tile too heavy for
// 32 bits, FP32 in the same words (FIXED picks one at compile time).  The
// fixed-point word is RN(v 2^e) from one FMA: with |v 2^e| <= 2^22, adding
// 1.5 2^23 rounds to an integer in the low mantissa bits (no F2I).
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kRoundMagicBits = 0x4B400000;
template <bool FIXED> __device__ __forceinline__ void region_add(int *reg, int idx, float v, float scale) {
    if (FIXED)
        red_shared_add_nc(reg + idx, __float_as_int(__fmaf_rn(v, scale, kRoundMagic)) - kRoundMagicBits);
    else
        red_shared_add_nc(reinterpret_cast<float *>(reg) + idx, v);
}

// largest 1-D weight of the window: NGP/CIC 1, TSC 3/4, PCS 2/3
template <int P> __device__ constexpr float window_wmax() { return P <= 2 ? 1.f : (P == 3 ? 0.75f : 0.6666667f); }

// first (unwrapped) stencil node of one axis, as in axis_first
template <int P> __device__ inline int axis_base(double g) {
    return (P % 2 == 0) ? (int)floor(g) - (P / 2 - 1) : (int)floor(__dadd_rn(g, 0.5)) - (P - 1) / 2;
}

// 1-D window of one axis: first (unwrapped) node and the P weights, computed
// exactly as axis_weights does.
template <int P> __device__ inline int axis_first(double g, float *w) {
    const int base = axis_base<P>(g);
#pragma unroll
    for (int o = 0; o < P; ++o) w[o] = (float)bspline<P>(__dsub_rn((double)(base + o), g));
    return base;
}

// Deposit into a shared region whose index 0 is the unwrapped node org.
template <int P, bool FIXED>
__device__ inline void deposit_region(int *reg, float scale, const int *org, double gx, double gy, double gz,
                                      float mass) {
    float wx[P], wy[P], wz[P];
    const int bx = axis_first<P>(gx, wx) - org[0];
    const int by = axis_first<P>(gy, wy) - org[1];
    const int bz = axis_first<P>(gz, wz) - org[2];
    const int base = (bx * kRegion + by) * kRegion + bz;
#pragma unroll
    for (int a = 0; a < P; ++a) {
#pragma unroll
        for (int b = 0; b < P; ++b) {
            const float wab = mass * wx[a] * wy[b];
#pragma unroll
            for (int c = 0; c < P; ++c) region_add<FIXED>(reg, base + (a * kRegion + b) * kRegion + c, wab * wz[c], scale);
        }
    }
}

// Region origin (unwrapped node of region index 0) for a particle at g:
// its base node b = floor(g) minus the offset of b inside its tile, minus 1.
__device__ inline int region_origin(double g, int n) {
    const int64_t b = (int64_t)floor(g);
    const int cw = wrapi(b, n);
    return (int)(b - (cw % kTile)) - 1;
}

template <typename T, int P>
__global__ void tile_paint_kernel(const double4 *__restrict__ sorted, const int *__restrict__ offset, int ntiles,
                                  int tpa, int n, T *mesh, T *mesh_shifted) {
    extern __shared__ int reg[];  // [2][kRegionCells]
    __shared__ int colc[kRegion * kRegion];
    __shared__ int wrap_t[3][kRegion];  // wrapped mesh index of each region index, per axis
    __shared__ unsigned s_mbits;
    __shared__ int s_cmax;
    const int nreg = mesh_shifted ? 2 : 1;
    const int lane = threadIdx.x & 31;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int p0 = offset[tile], p1 = offset[tile + 1];
        if (p0 == p1) continue;
        __syncthreads();
        for (int i = threadIdx.x; i < nreg * kRegionCells; i += blockDim.x) reg[i] = 0;
        for (int i = threadIdx.x; i < kRegion * kRegion; i += blockDim.x) colc[i] = 0;
        if (threadIdx.x == 0) s_mbits = 0u, s_cmax = 0;
        if (threadIdx.x < 3 * kRegion) {
            // region origin of this tile: tile origin - 1
            const int ax = threadIdx.x / kRegion, ri = threadIdx.x % kRegion;
            const int tcoord = ax == 0 ? tile / (tpa * tpa) : (ax == 1 ? (tile / tpa) % tpa : tile % tpa);
            wrap_t[ax][ri] = wrapi((int64_t)tcoord * kTile - 1 + ri, n);
        }
        __syncthreads();
        // bound of any node's sum: particles per first-node column, max |mass|
        float mloc = 0.f;
        for (int i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
            const double4 q = sorted[i];
            const int fx = axis_base<P>(q.x) - region_origin(q.x, n);
            const int fy = axis_base<P>(q.y) - region_origin(q.y, n);
            atomicAdd(&colc[fx * kRegion + fy], 1);
            mloc = fmaxf(mloc, fabsf((float)q.w));
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) mloc = fmaxf(mloc, __shfl_xor_sync(0xffffffffu, mloc, o));
        if (lane == 0) atomicMax(&s_mbits, __float_as_uint(mloc));  // non-negative floats order as integers
        __syncthreads();
        int cm = 0;
        for (int c = threadIdx.x; c < kRegion * kRegion; c += blockDim.x) {
            const int x = c / kRegion, y = c % kRegion;
            int sum = 0;
            for (int dx = 0; dx <= P && dx <= x; ++dx)
                for (int dy = 0; dy <= P && dy <= y; ++dy) sum += colc[(x - dx) * kRegion + (y - dy)];
            cm = max(cm, sum);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) cm = max(cm, __shfl_xor_sync(0xffffffffu, cm, o));
        if (lane == 0) atomicMax(&s_cmax, cm);
        __syncthreads();
        constexpr float wa = window_wmax<P>();
        // (1 + 2^-20): FP32 products of rounded weights may exceed wmax^3 by a few ulps
        const double bound =
            (double)s_cmax * (double)__uint_as_float(s_mbits) * (double)(wa * wa * wa) * (1.0 + 0x1p-20);
        // rounding adds at most 1/2 per deposit, one deposit per particle of the window;
        // one deposit stays within 2^22 (region_add's rounding)
        const double room = 2147483647.0 - (double)s_cmax;
        const double one = (double)__uint_as_float(s_mbits) * (double)(wa * wa * wa) * (1.0 + 0x1p-20);
        int e = 100;
        if (bound > 0.0) e = min(100, min(ilogb(room / bound), ilogb(4194304.0 / one)));
        const float scale = ldexpf(1.f, e);
        const bool fixed = s_cmax <= 65536;
        auto deposit_all = [&](auto fixed_tag) {
            constexpr bool F = decltype(fixed_tag)::value;
            for (int i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
                const double4 q = sorted[i];
                int org[3] = {region_origin(q.x, n), region_origin(q.y, n), region_origin(q.z, n)};
                deposit_region<P, F>(reg, scale, org, q.x, q.y, q.z, (float)q.w);
                if (mesh_shifted)
                    deposit_region<P, F>(reg + kRegionCells, scale, org, __dadd_rn(q.x, 0.5), __dadd_rn(q.y, 0.5),
                                         __dadd_rn(q.z, 0.5), (float)q.w);
            }
        };
        if (fixed)
            deposit_all(std::true_type{});
        else
            deposit_all(std::false_type{});
        __syncthreads();
        const double unscale = ldexp(1.0, -e);
        for (int i = threadIdx.x; i < nreg * kRegionCells; i += blockDim.x) {
            const int word = reg[i];
            if (word == 0) continue;
            const float v = fixed ? (float)((double)word * unscale) : __int_as_float(word);
            const int r = i % kRegionCells;
            const int rz = r % kRegion, ry = (r / kRegion) % kRegion, rx = r / (kRegion * kRegion);
            const size_t cell = ((size_t)wrap_t[0][rx] * n + wrap_t[1][ry]) * n + wrap_t[2][rz];
            atomicAdd((i < kRegionCells ? mesh : mesh_shifted) + cell, (T)v);
        }
    }
}

// ------------------------------------------------- compact-record tiled paint
// For windows of order 2..4 (continuous weights) the sort writes a 16-byte
// record per particle instead of its FP64 grid coordinates: the FP32
// fraction of the window argument per axis (g - floor(g) for even orders,
// (g + 1/2) - floor(g + 1/2) for odd ones) and the first stencil node of both
// grids relative to the tile's region, packed in 5 bits per axis.  Node
// selection stays FP64-exact (made in the sort); the 1-D weights are the
// window polynomials of the fraction in FP32 (the per-particle kernel rounds
// its FP64 weights to FP32 for FP32 meshes; both are within a few FP32 ulps).
// The +1/2-shifted grid's fraction is f + 1/2 - (its first node - the plain
// grid's first node).  Weights other than 1 travel in a separate FP32 array.
struct __align__(16) PaintRec {
    float fx, fy, fz;
    uint32_t nodes;  // plain grid x, y, z then shifted grid x, y, z: 5 bits each
};

template <int P> __device__ inline double window_arg(double g) { return (P % 2 == 0) ? g : __dadd_rn(g, 0.5); }

template <int P>
__global__ void tile_scatter_rec_kernel(const double *__restrict__ pos, const double *__restrict__ weight,
                                        int64_t np, int n, Frame scale, const int *tile_of, int *cursor,
                                        PaintRec *sorted, float *sorted_w) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride) {
        double g[3];
        grid_coords(pos, i, scale, g);
        const int tid = tile_of[i];
        const unsigned same = __match_any_sync(__activemask(), tid);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(same) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&cursor[tid], __popc(same));
        base = __shfl_sync(same, base, leader);
        const int slot = base + __popc(same & ((1u << lane) - 1));
        PaintRec r;
        float f[3];
        uint32_t nodes = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int org = region_origin(g[d], n);
            const double a = window_arg<P>(g[d]);
            const double fl = floor(a);
            f[d] = (float)__dsub_rn(a, fl);
            const uint32_t b0 = (uint32_t)(axis_base<P>(g[d]) - org);
            const uint32_t b1 = (uint32_t)(axis_base<P>(__dadd_rn(g[d], 0.5)) - org);
            nodes |= b0 << (5 * d);
            nodes |= b1 << (15 + 5 * d);
        }
        r.fx = f[0], r.fy = f[1], r.fz = f[2];
        r.nodes = nodes;
        sorted[slot] = r;
        if (sorted_w) sorted_w[slot] = (float)mass_of(weight, i, scale);
    }
}

// 1-D weights of the nodes first .. first + P - 1 from the window fraction f
template <int P> __device__ __forceinline__ void window_weights_f32(float f, float *w) {
    if (P == 2) {
        w[0] = 1.f - f;
        w[1] = f;
    } else if (P == 3) {
        const float h = 0.5f - f, u = 1.f - f;
        w[0] = 0.5f * u * u;
        w[1] = 0.75f - h * h;
        w[2] = 0.5f * f * f;
    } else {  // P == 4
        const float u = 1.f - f, f2 = f * f, u2 = u * u;
        constexpr float s6 = 1.f / 6.f;
        w[0] = s6 * u2 * u;
        w[1] = s6 * (4.f - 6.f * f2 + 3.f * f2 * f);
        w[2] = s6 * (4.f - 6.f * u2 + 3.f * u2 * u);
        w[3] = s6 * f2 * f;
    }
}

template <int P, bool FIXED>
__device__ __forceinline__ void deposit_rec(int *reg, float scale, uint32_t bx, uint32_t by, uint32_t bz, float fx,
                                            float fy, float fz, float mass) {
    float wx[P], wy[P], wz[P];
    window_weights_f32<P>(fx, wx);
    window_weights_f32<P>(fy, wy);
    window_weights_f32<P>(fz, wz);
    const int base = ((int)bx * kRegion + (int)by) * kRegion + (int)bz;
#pragma unroll
    for (int a = 0; a < P; ++a) {
#pragma unroll
        for (int b = 0; b < P; ++b) {
            const float wab = mass * wx[a] * wy[b];
#pragma unroll
            for (int c = 0; c < P; ++c) region_add<FIXED>(reg, base + (a * kRegion + b) * kRegion + c, wab * wz[c], scale);
        }
    }
}

// region_out != nullptr: each tile writes its whole region (both grids, FP32
// values) to region_out[tile] with plain stores and tile_gather_kernel sums
// every node's contributions in a fixed order (bitwise reproducible meshes);
// otherwise the regions are added to the mesh with atomics.
template <typename T, int P>
__global__ void tile_paint_rec_kernel(const PaintRec *__restrict__ sorted, const float *__restrict__ sorted_w,
                                      float mass_const, const int *__restrict__ offset, int ntiles, int tpa, int n,
                                      T *mesh, T *mesh_shifted, float *__restrict__ region_out) {
    extern __shared__ int reg[];  // [2][kRegionCells]
    __shared__ int colc[kRegion * kRegion];
    __shared__ int wrap_t[3][kRegion];
    __shared__ unsigned s_mbits;
    __shared__ int s_cmax;
    const int nreg = mesh_shifted ? 2 : 1;
    const int lane = threadIdx.x & 31;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int p0 = offset[tile], p1 = offset[tile + 1];
        if (p0 == p1) {
            if (region_out)  // the gather reads every tile's region
                for (int i = threadIdx.x; i < nreg * kRegionCells; i += blockDim.x)
                    region_out[(size_t)tile * nreg * kRegionCells + i] = 0.f;
            continue;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nreg * kRegionCells; i += blockDim.x) reg[i] = 0;
        for (int i = threadIdx.x; i < kRegion * kRegion; i += blockDim.x) colc[i] = 0;
        if (threadIdx.x == 0) s_mbits = 0u, s_cmax = 0;
        if (threadIdx.x < 3 * kRegion) {
            const int ax = threadIdx.x / kRegion, ri = threadIdx.x % kRegion;
            const int tcoord = ax == 0 ? tile / (tpa * tpa) : (ax == 1 ? (tile / tpa) % tpa : tile % tpa);
            wrap_t[ax][ri] = wrapi((int64_t)tcoord * kTile - 1 + ri, n);
        }
        __syncthreads();
        // bound of any node's sum: particles per first-node column, max |mass|
        float mloc = sorted_w ? 0.f : fabsf(mass_const);
        for (int i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
            const uint32_t nodes = sorted[i].nodes;
            atomicAdd(&colc[(int)(nodes & 31u) * kRegion + (int)((nodes >> 5) & 31u)], 1);
            if (sorted_w) mloc = fmaxf(mloc, fabsf(sorted_w[i]));
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) mloc = fmaxf(mloc, __shfl_xor_sync(0xffffffffu, mloc, o));
        if (lane == 0) atomicMax(&s_mbits, __float_as_uint(mloc));
        __syncthreads();
        int cm = 0;
        for (int c = threadIdx.x; c < kRegion * kRegion; c += blockDim.x) {
            const int x = c / kRegion, y = c % kRegion;
            int sum = 0;
            for (int dx = 0; dx <= P && dx <= x; ++dx)
                for (int dy = 0; dy <= P && dy <= y; ++dy) sum += colc[(x - dx) * kRegion + (y - dy)];
            cm = max(cm, sum);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) cm = max(cm, __shfl_xor_sync(0xffffffffu, cm, o));
        if (lane == 0) atomicMax(&s_cmax, cm);
        __syncthreads();
        constexpr float wa = window_wmax<P>();
        // FP32 weights may exceed wmax^3 by a few ulps: slack (1 + 2^-20)
        const double one = (double)__uint_as_float(s_mbits) * (double)(wa * wa * wa) * (1.0 + 0x1p-20);
        const double bound = (double)s_cmax * one;
        const double room = 2147483647.0 - (double)s_cmax;
        int e = 100;
        if (bound > 0.0) e = min(100, min(ilogb(room / bound), ilogb(4194304.0 / one)));
        const float scale = ldexpf(1.f, e);
        const bool fixed = s_cmax <= 65536;
        auto deposit_all = [&](auto fixed_tag) {
            constexpr bool F = decltype(fixed_tag)::value;
            for (int i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
                const PaintRec r = sorted[i];
                const float m = sorted_w ? sorted_w[i] : mass_const;
                deposit_rec<P, F>(reg, scale, r.nodes & 31u, (r.nodes >> 5) & 31u, (r.nodes >> 10) & 31u, r.fx, r.fy,
                                  r.fz, m);
                if (mesh_shifted) {
                    const uint32_t b1x = (r.nodes >> 15) & 31u, b1y = (r.nodes >> 20) & 31u, b1z = (r.nodes >> 25) & 31u;
                    const float gx = r.fx + 0.5f - (float)((int)b1x - (int)(r.nodes & 31u));
                    const float gy = r.fy + 0.5f - (float)((int)b1y - (int)((r.nodes >> 5) & 31u));
                    const float gz = r.fz + 0.5f - (float)((int)b1z - (int)((r.nodes >> 10) & 31u));
                    deposit_rec<P, F>(reg + kRegionCells, scale, b1x, b1y, b1z, gx, gy, gz, m);
                }
            }
        };
        if (fixed)
            deposit_all(std::true_type{});
        else
            deposit_all(std::false_type{});
        __syncthreads();
        const double unscale = ldexp(1.0, -e);
        if (region_out) {
            float *dst = region_out + (size_t)tile * nreg * kRegionCells;
            for (int i = threadIdx.x; i < nreg * kRegionCells; i += blockDim.x) {
                const int word = reg[i];
                dst[i] = fixed ? (float)((double)word * unscale) : __int_as_float(word);
            }
            continue;
        }
        for (int i = threadIdx.x; i < nreg * kRegionCells; i += blockDim.x) {
            const int word = reg[i];
            if (word == 0) continue;
            const float v = fixed ? (float)((double)word * unscale) : __int_as_float(word);
            const int r = i % kRegionCells;
            const int rz = r % kRegion, ry = (r / kRegion) % kRegion, rx = r / (kRegion * kRegion);
            const size_t cell = ((size_t)wrap_t[0][rx] * n + wrap_t[1][ry]) * n + wrap_t[2][rz];
            atomicAdd((i < kRegionCells ? mesh : mesh_shifted) + cell, (T)v);
        }
    }
}

// The node at local coordinate l (0..15) of a tile along one axis lies in
// the regions of (at most) the previous tile at region index l + 17 (when
// l <= 2), the tile itself at l + 1, and the next tile at 0 (when l == 15);
// dt = -1, 0, +1 in that fixed order.
__device__ __forceinline__ int covering(int l, int *dt, int *ri) {
    int k = 0;
    if (l <= 2) dt[k] = -1, ri[k++] = l + kTile + 1;
    dt[k] = 0, ri[k++] = l + 1;
    if (l == kTile - 1) dt[k] = 1, ri[k++] = 0;
    return k;
}

// mesh[node] (+)= the node's contributions from every tile region covering
// it (empty tiles have zero regions), summed in a fixed order: the node's own
// x line of each covering (y, z) tile first, then the previous and the next
// x tile.  One block per (tile core, grid); thread (ly, lz) holds the 16 nodes
// of its x line, so the loads of the dominant term are independent.
template <typename T>
__global__ void __launch_bounds__(256) tile_gather_kernel(const float *__restrict__ region, int tpa, int n, int nreg,
                                                          int accumulate, T *mesh, T *mesh_shifted) {
    const int ntiles = tpa * tpa * tpa;
    const int ly = threadIdx.x >> 4, lz = threadIdx.x & 15;
    int dy[2], ry[2], dz[2], rz[2];
    const int ny = covering(ly, dy, ry), nz = covering(lz, dz, rz);
    for (int w = blockIdx.x; w < ntiles * nreg; w += gridDim.x) {
        const int k = w / ntiles, tile = w - k * ntiles;
        const int tx = tile / (tpa * tpa), ty = (tile / tpa) % tpa, tz = tile % tpa;
        auto base = [&](int cx, int b, int d) {
            const int t = (cx * tpa + (ty + dy[b] + tpa) % tpa) * tpa + (tz + dz[d] + tpa) % tpa;
            return region + ((size_t)t * nreg + k) * kRegionCells + ry[b] * kRegion + rz[d];
        };
        float acc[kTile];
#pragma unroll
        for (int lx = 0; lx < kTile; ++lx) acc[lx] = 0.f;
        for (int b = 0; b < ny; ++b)
            for (int d = 0; d < nz; ++d) {
                const float *r = base(tx, b, d);
#pragma unroll
                for (int lx = 0; lx < kTile; ++lx) acc[lx] += __ldg(r + (lx + 1) * kRegion * kRegion);
            }
        const int px = tx == 0 ? tpa - 1 : tx - 1, nxt = tx + 1 == tpa ? 0 : tx + 1;
        for (int b = 0; b < ny; ++b)
            for (int d = 0; d < nz; ++d) {
                const float *r = base(px, b, d);
#pragma unroll
                for (int lx = 0; lx < 3; ++lx) acc[lx] += __ldg(r + (lx + kTile + 1) * kRegion * kRegion);
                acc[kTile - 1] += __ldg(base(nxt, b, d));
            }
        T *m = (k == 0 ? mesh : mesh_shifted) + ((size_t)(tx * kTile) * n + (ty * kTile + ly)) * n + (tz * kTile + lz);
#pragma unroll
        for (int lx = 0; lx < kTile; ++lx) {
            T *dst = m + (size_t)lx * n * n;
            *dst = accumulate ? *dst + (T)acc[lx] : (T)acc[lx];
        }
    }
}

template <typename T>
static int launch_tiled(cnpc_ctx *ctx, const double *pos, const double *w, int64_t np, int n, const Frame &scale,
                        int window, T *m1, T *m2, int accumulate, cudaStream_t s) {
    const int tpa = (n + kTile - 1) / kTile;
    const int nt = tpa * tpa * tpa;
    const size_t off_counts = 0, off_offset = off_counts + sizeof(int) * nt,
                 off_cursor = off_offset + sizeof(int) * (nt + 1), off_tile = off_cursor + sizeof(int) * nt;
    size_t off_sorted = off_tile + sizeof(int) * (size_t)np;
    off_sorted = (off_sorted + 255) / 256 * 256;
    const size_t bytes = off_sorted + sizeof(double4) * (size_t)np;
    int st = ensure_buffer(ctx, &ctx->paint_ws, &ctx->paint_ws_bytes, bytes, s);
    if (st) return st;
    char *ws = static_cast<char *>(ctx->paint_ws);
    int *count = reinterpret_cast<int *>(ws + off_counts);
    int *offset = reinterpret_cast<int *>(ws + off_offset);
    int *cursor = reinterpret_cast<int *>(ws + off_cursor);
    int *tile_of = reinterpret_cast<int *>(ws + off_tile);
    double4 *sorted = reinterpret_cast<double4 *>(ws + off_sorted);
    st = check_cuda(ctx, cudaMemsetAsync(count, 0, sizeof(int) * nt, s), "memset tile counts");
    if (st) return st;
    const int threads = 256;
    const int pblocks = (int)std::min<int64_t>((np + threads - 1) / threads, (int64_t)ctx->num_sms * 16);
    tile_count_kernel<<<pblocks, threads, 0, s>>>(pos, np, n, scale, tpa, count, tile_of);
    tile_scan_kernel<<<1, 1024, 0, s>>>(count, nt, offset, cursor);
    if (window >= 2 && std::is_same<T, float>::value) {
        // compact records: 16 bytes per particle (+4 with weights) in the
        // space of the FP64 records
        PaintRec *rec = reinterpret_cast<PaintRec *>(sorted);
        float *rec_w = w ? reinterpret_cast<float *>(rec + np) : nullptr;
        const size_t smem = sizeof(int) * kRegionCells * (m2 ? 2 : 1);
        const int tblocks = (int)std::min<int64_t>(nt, (int64_t)ctx->num_sms * 8);
        // regions through a buffer and a fixed-order gather when the tiles
        // cover the mesh exactly (n a multiple of 16), atomics otherwise
        float *region = nullptr;
        const int nreg = m2 ? 2 : 1;
        if (n % kTile == 0) {
            st = ensure_buffer(ctx, &ctx->aux, &ctx->aux_bytes, sizeof(float) * (size_t)nt * nreg * kRegionCells, s);
            if (st) return st;
            region = static_cast<float *>(ctx->aux);
        }
        switch (window) {
#define CNPC_TPR(P_)                                                                                          \
    case P_:                                                                                                  \
        tile_scatter_rec_kernel<P_><<<pblocks, threads, 0, s>>>(pos, w, np, n, scale, tile_of, cursor, rec, rec_w); \
        st = check_cuda(ctx, cudaFuncSetAttribute(tile_paint_rec_kernel<T, P_>,                               \
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),    \
                        "tile paint smem");                                                                   \
        if (st) return st;                                                                                    \
        tile_paint_rec_kernel<T, P_><<<tblocks, 256, smem, s>>>(rec, rec_w, (float)scale.mass_scale, offset, nt, \
                                                                tpa, n, m1, m2, region);                      \
        break;
            CNPC_TPR(2) CNPC_TPR(3) CNPC_TPR(4)
#undef CNPC_TPR
            default: return fail(ctx, CNPC_EINVAL, "window must be 1..4");
        }
        st = check_launch(ctx, "tile_paint_rec_kernel");
        if (st || !region) return st;
        const int gblocks = (int)std::min<int64_t>((int64_t)nt * nreg, (int64_t)ctx->num_sms * 8);
        tile_gather_kernel<T><<<gblocks, 256, 0, s>>>(region, tpa, n, nreg, accumulate, m1, m2);
        return check_launch(ctx, "tile_gather_kernel");
    }
    tile_scatter_kernel<<<pblocks, threads, 0, s>>>(pos, w, np, scale, tile_of, cursor, sorted);
    st = check_launch(ctx, "tile sort");
    if (st) return st;
    const size_t smem = sizeof(int) * kRegionCells * (m2 ? 2 : 1);
    const int tblocks = (int)std::min<int64_t>(nt, (int64_t)ctx->num_sms * 8);
    switch (window) {
#define CNPC_TP(P_)                                                                                        \
    case P_:                                                                                               \
        st = check_cuda(ctx, cudaFuncSetAttribute(tile_paint_kernel<T, P_>,                                \
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), \
                        "tile paint smem");                                                                \
        if (st) return st;                                                                                 \
        tile_paint_kernel<T, P_><<<tblocks, 256, smem, s>>>(sorted, offset, nt, tpa, n, m1, m2);           \
        break;
        CNPC_TP(1) CNPC_TP(2) CNPC_TP(3) CNPC_TP(4)
#undef CNPC_TP
        default: return fail(ctx, CNPC_EINVAL, "window must be 1..4");
    }
    return check_launch(ctx, "tile_paint_kernel");
}

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_paint_ex(cnpc_ctx *ctx, int dtype, const double *d_pos, const double *d_weight,
                             int64_t np, int n, double boxsize, int window, const double *h_origin,
                             double mass_scale, int accumulate, void *d_mesh, void *d_mesh_shifted,
                             cnpc_stream_t stream) {
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
    int st;
    // the tiled FP32 paint of windows 2..4 on a multiple of 16 writes every node
    // itself (fixed-order gather of the tile regions): no zeroing needed
    const bool tiled = dtype == CNPC_F32 && n >= 2 * kTile && np >= 8 * (int64_t)n * n * n / 64;
    const bool gathered = tiled && window >= 2 && n % kTile == 0;
    if (!accumulate && !gathered) {
        st = check_cuda(ctx, cudaMemsetAsync(d_mesh, 0, cells * esz, s), "memset mesh");
        if (st) return st;
        if (d_mesh_shifted) {
            st = check_cuda(ctx, cudaMemsetAsync(d_mesh_shifted, 0, cells * esz, s), "memset mesh");
            if (st) return st;
        }
    }
    if (np == 0) return CNPC_OK;
    Frame f;
    f.ox = h_origin ? h_origin[0] : 0.0;
    f.oy = h_origin ? h_origin[1] : 0.0;
    f.oz = h_origin ? h_origin[2] : 0.0;
    f.scale = (double)n / boxsize;
    f.mass_scale = mass_scale;
    // the tiled deposit pays off once tiles hold many particles; its FP32
    // shared-memory region would round FP64 meshes, so FP64 stays per particle
    if (dtype == CNPC_F32) {
        if (tiled)
            return launch_tiled<float>(ctx, d_pos, d_weight, np, n, f, window, (float *)d_mesh,
                                       (float *)d_mesh_shifted, accumulate, s);
        return launch_paint<float>(ctx, d_pos, d_weight, np, n, f, window, (float *)d_mesh,
                                   (float *)d_mesh_shifted, s);
    }
    return launch_paint<double>(ctx, d_pos, d_weight, np, n, f, window, (double *)d_mesh,
                                (double *)d_mesh_shifted, s);
}

extern "C" int cnpc_paint(cnpc_ctx *ctx, int dtype, const double *d_pos, const double *d_weight,
                          int64_t np, int n, double boxsize, int window, void *d_mesh,
                          void *d_mesh_shifted, cnpc_stream_t stream) {
    return cnpc_paint_ex(ctx, dtype, d_pos, d_weight, np, n, boxsize, window, nullptr, 1.0, 0, d_mesh,
                         d_mesh_shifted, stream);
}
