// Box-geometry catalogs read from FITS or HDF5 files: the position, velocity
// and weight columns decoded on the device, with the redshift-space shift of
// catalog_processor.py:648-693 (add_rsd, box-like branch) applied there.
//
// A column is a strided run of scalars in device memory (the raw rows of a
// FITS binary table, big-endian, or one contiguous HDF5 dataset), so both
// formats reach the kernel without a host-side decode.  The shift is
//   x_d <- (x_d + (f los_d) v_d) mod L,   f = (1 + z) / (100 E(z)),
// with the reference's elementwise product of the line-of-sight vector and
// the velocity, each operation rounded separately as numpy does it, and the
// result wrapped with numpy's float remainder (fmod, then + L where the sign
// differs from L's).
#include <cmath>

#include "internal.h"

namespace cnpc {

namespace {

struct BoxParams {
    cnpc_colref col[CNPC_BOX_NCOLS];
    int apply_rsd;
    double shift[3];  // f * los_d, rounded on the host as numpy rounds it
    double box_length;
};

__device__ inline double read_ref(const cnpc_colref &c, int64_t i) {
    const uint8_t *p = static_cast<const uint8_t *>(c.d_base) + i * c.stride;
    int nb;
    switch (c.type) {
        case CNPC_CT_F32: case CNPC_CT_I32: nb = 4; break;
        case CNPC_CT_I16: nb = 2; break;
        case CNPC_CT_U8: case CNPC_CT_BOOL: nb = 1; break;
        default: nb = 8;
    }
    uint64_t u = 0;
    if (c.big_endian) {
        for (int k = 0; k < nb; ++k) u = (u << 8) | (uint64_t)p[k];
    } else {
        for (int k = nb - 1; k >= 0; --k) u = (u << 8) | (uint64_t)p[k];
    }
    double v;
    switch (c.type) {
        case CNPC_CT_F64: v = __longlong_as_double((long long)u); break;
        case CNPC_CT_F32: v = (double)__int_as_float((int)(uint32_t)u); break;
        case CNPC_CT_I16: v = (double)(int16_t)(uint16_t)u; break;
        case CNPC_CT_I32: v = (double)(int32_t)(uint32_t)u; break;
        case CNPC_CT_I64: v = (double)(long long)u; break;
        case CNPC_CT_U8: v = (double)u; break;
        case CNPC_CT_BOOL: v = (u == (uint64_t)'T' || u == 1u) ? 1.0 : 0.0; break;
        default: v = 0.0;
    }
    if (c.scale != 1.0 || c.zero != 0.0) v = __dadd_rn(c.zero, __dmul_rn(c.scale, v));
    return v;
}

// numpy's float remainder a % b for b > 0
__device__ inline double py_mod(double a, double b) {
    double m = fmod(a, b);
    if (m != 0.0) {
        if ((m < 0.0) != (b < 0.0)) m = __dadd_rn(m, b);
    } else {
        m = copysign(0.0, b);
    }
    return m;
}

__global__ void box_catalog_kernel(int64_t nrows, const BoxParams P, double *__restrict__ pos,
                                   double *__restrict__ weight) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += stride) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const cnpc_colref &c = P.col[CNPC_BOX_X + d];
            double x = c.type == CNPC_CT_ABSENT ? 0.0 : read_ref(c, i);
            if (P.apply_rsd) {
                const double v = read_ref(P.col[CNPC_BOX_VX + d], i);
                x = py_mod(__dadd_rn(x, __dmul_rn(P.shift[d], v)), P.box_length);
            }
            pos[3 * i + d] = x;
        }
        const cnpc_colref &w = P.col[CNPC_BOX_W];
        weight[i] = w.type == CNPC_CT_ABSENT ? 1.0 : read_ref(w, i);
    }
}

}  // namespace

}  // namespace cnpc

using namespace cnpc;

extern "C" int cnpc_box_catalog(cnpc_ctx *ctx, int64_t nrows, const cnpc_colref *h_cols, int apply_rsd,
                                const double *h_shift, double box_length, double *d_pos, double *d_weight,
                                cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, nrows >= 0, "negative row count");
    CNPC_REQUIRE(ctx, h_cols != nullptr, "null column table");
    CNPC_REQUIRE(ctx, nrows == 0 || (d_pos && d_weight), "null output");
    BoxParams P;
    for (int k = 0; k < CNPC_BOX_NCOLS; ++k) {
        const cnpc_colref &c = h_cols[k];
        CNPC_REQUIRE(ctx, c.type >= CNPC_CT_ABSENT && c.type <= CNPC_CT_BOOL, "bad column type");
        CNPC_REQUIRE(ctx, c.type == CNPC_CT_ABSENT || nrows == 0 || c.d_base != nullptr, "null column");
        P.col[k] = c;
    }
    P.apply_rsd = apply_rsd ? 1 : 0;
    if (P.apply_rsd) {
        CNPC_REQUIRE(ctx, h_shift != nullptr, "null RSD shift");
        CNPC_REQUIRE(ctx, box_length > 0.0, "box length must be positive");
        for (int d = 0; d < 3; ++d) {
            CNPC_REQUIRE(ctx, h_cols[CNPC_BOX_VX + d].type != CNPC_CT_ABSENT, "RSD needs the velocity columns");
            P.shift[d] = h_shift[d];
        }
    }
    P.box_length = box_length;
    if (nrows == 0) return CNPC_OK;
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((nrows + threads - 1) / threads, (int64_t)ctx->num_sms * 8);
    box_catalog_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(nrows, P, d_pos, d_weight);
    return check_launch(ctx, "box_catalog_kernel");
}
