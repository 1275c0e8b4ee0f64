// Context, error reporting and cuFFT plan cache.
#include <cstdio>
#include <stdexcept>

#include "internal.h"

namespace cnpc {

int fail(cnpc_ctx *ctx, int status, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

int check_cuda(cnpc_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CNPC_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(ctx, CNPC_ENOMEM, std::string(what) + ": " + cudaGetErrorString(e));
    }
    return fail(ctx, CNPC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_launch(cnpc_ctx *ctx, const char *what) {
    return check_cuda(ctx, cudaGetLastError(), what);
}

int ensure_buffer(cnpc_ctx *ctx, void **buf, size_t *have, size_t bytes, cudaStream_t stream) {
    if (*have >= bytes) return CNPC_OK;
    if (*buf) {
        // the previous buffer may still be in use by work queued on `stream`
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return check_cuda(ctx, e, "workspace sync");
        cudaFree(*buf);
        *buf = nullptr;
        *have = 0;
    }
    size_t want = bytes < (size_t)(1 << 20) ? (size_t)(1 << 20) : bytes;
    cudaError_t e = cudaMalloc(buf, want);
    if (e != cudaSuccess) return check_cuda(ctx, e, "workspace alloc");
    *have = want;
    return CNPC_OK;
}

int ensure_scratch(cnpc_ctx *ctx, size_t bytes, cudaStream_t stream) {
    return ensure_buffer(ctx, &ctx->scratch, &ctx->scratch_bytes, bytes, stream);
}

int ensure_status(cnpc_ctx *ctx) {
    if (ctx->d_status) return CNPC_OK;
    int *p = nullptr;
    cudaError_t e = cudaMalloc(&p, 256);
    if (e != cudaSuccess) return check_cuda(ctx, e, "status word alloc");
    e = cudaMemset(p, 0, 256);
    if (e != cudaSuccess) {
        cudaFree(p);
        return check_cuda(ctx, e, "status word clear");
    }
    ctx->d_status = p;
    return CNPC_OK;
}

// The plan of (type, n, batch, real_dist), made on first use, with the shared
// work area of the context grown to its needs and attached, and the stream set.
static int get_plan(cnpc_ctx *ctx, cufftType type, int n, int batch, long long real_dist, cudaStream_t stream,
                    cufftHandle *out) {
    auto key = std::make_tuple((int)type, n, batch, real_dist);
    auto it = ctx->plans.find(key);
    if (it == ctx->plans.end()) {
        // 64-bit plan sizes: a batch of 16 fields of 512^3 holds 2^31 elements,
        // which the 32-bit cufftPlanMany rejects (CUFFT_INTERNAL_ERROR)
        cufftHandle h;
        cufftResult r = cufftCreate(&h);
        if (r != CUFFT_SUCCESS)
            return fail(ctx, CNPC_ECUFFT, "cufftCreate failed with code " + std::to_string((int)r));
        r = cufftSetAutoAllocation(h, 0);
        long long dims[3] = {n, n, n};
        long long real_embed[3] = {n, n, n};
        long long spec_embed[3] = {n, n, n / 2 + 1};
        const long long spec_dist = (long long)n * n * (n / 2 + 1);
        const bool forward = type == CUFFT_R2C || type == CUFFT_D2Z;
        size_t work = 0;
        if (r == CUFFT_SUCCESS) {
            if (forward)
                r = cufftMakePlanMany64(h, 3, dims, real_embed, 1, real_dist, spec_embed, 1, spec_dist, type, batch,
                                        &work);
            else
                r = cufftMakePlanMany64(h, 3, dims, spec_embed, 1, spec_dist, real_embed, 1, real_dist, type, batch,
                                        &work);
        }
        if (r != CUFFT_SUCCESS) {
            cufftDestroy(h);
            if (r == CUFFT_ALLOC_FAILED) return fail(ctx, CNPC_ENOMEM, "cufftMakePlanMany64: allocation failed");
            return fail(ctx, CNPC_ECUFFT, "cufftMakePlanMany64 failed with code " + std::to_string((int)r));
        }
        it = ctx->plans.emplace(key, cnpc_ctx::FftPlan{h, work}).first;
    }
    const cnpc_ctx::FftPlan &p = it->second;
    int st = ensure_buffer(ctx, &ctx->fft_ws, &ctx->fft_ws_bytes, p.work, stream);
    if (st) return st;
    cufftResult r = cufftSetWorkArea(p.h, ctx->fft_ws);
    if (r == CUFFT_SUCCESS) r = cufftSetStream(p.h, stream);
    if (r != CUFFT_SUCCESS) return fail(ctx, CNPC_ECUFFT, "cufft work area / stream: code " + std::to_string((int)r));
    *out = p.h;
    return CNPC_OK;
}

}  // namespace cnpc

using namespace cnpc;

extern "C" {

int cnpc_version(void) { return 100; }

const char *cnpc_status_string(int status) {
    switch (status) {
        case CNPC_OK: return "ok";
        case CNPC_EINVAL: return "invalid argument";
        case CNPC_ENOMEM: return "out of device memory";
        case CNPC_ECUDA: return "CUDA error";
        case CNPC_ECUFFT: return "cuFFT error";
        case CNPC_ETIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

int cnpc_ctx_create(cnpc_ctx **ctx, int device) {
    if (!ctx) return CNPC_EINVAL;
    *ctx = nullptr;
    cnpc_ctx *c = new (std::nothrow) cnpc_ctx();
    if (!c) return CNPC_ENOMEM;
    c->device = device;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        delete c;
        return CNPC_ECUDA;
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete c;
        return CNPC_ECUDA;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
        c->num_sms = sms;
    *ctx = c;
    return CNPC_OK;
}

int cnpc_ctx_destroy(cnpc_ctx *ctx) {
    if (!ctx) return CNPC_OK;
    for (auto &kv : ctx->plans) cufftDestroy(kv.second.h);
    if (ctx->fft_ws) cudaFree(ctx->fft_ws);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->paint_ws) cudaFree(ctx->paint_ws);
    if (ctx->aux) cudaFree(ctx->aux);
    if (ctx->shell_ws) cudaFree(ctx->shell_ws);
    if (ctx->d_status) cudaFree(ctx->d_status);
    delete ctx;
    return CNPC_OK;
}

const char *cnpc_ctx_last_error(cnpc_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int cnpc_ctx_set_wait_limit(cnpc_ctx *ctx, int64_t polls) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, polls >= 0, "wait limit must be >= 0");
    ctx->wait_limit = polls;
    return CNPC_OK;
}

int cnpc_ctx_take_status(cnpc_ctx *ctx, cnpc_stream_t stream, int *h_status) {
    CNPC_REQUIRE(ctx, ctx != nullptr, "null context");
    CNPC_REQUIRE(ctx, h_status != nullptr, "null status pointer");
    *h_status = CNPC_OK;
    if (!ctx->d_status) return CNPC_OK;  // no bounded wait has run in this context
    cudaStream_t s = (cudaStream_t)stream;
    int v = 0;
    int st = check_cuda(ctx, cudaMemcpyAsync(&v, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, s),
                        "status word read");
    if (st) return st;
    st = check_cuda(ctx, cudaStreamSynchronize(s), "status word read");
    if (st) return st;
    st = check_cuda(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s), "status word clear");
    if (st) return st;
    *h_status = v;
    return CNPC_OK;
}

int cnpc_fft_r2c(cnpc_ctx *ctx, int dtype, int n, int batch, const void *d_real, int64_t real_dist,
                 void *d_spec, cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, n >= 2 && n % 2 == 0 && n <= 2048, "n must be even, 2..2048");
    CNPC_REQUIRE(ctx, batch >= 1, "batch must be >= 1");
    CNPC_REQUIRE(ctx, d_real && d_spec, "null buffer");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    cufftHandle h;
    const long long cells = (long long)n * n * n;
    CNPC_REQUIRE(ctx, real_dist == 0 || real_dist >= cells, "real_dist must be 0 or >= n^3");
    CNPC_REQUIRE(ctx, real_dist < (1ll << 31), "real_dist too large");
    int st = get_plan(ctx, dtype == CNPC_F32 ? CUFFT_R2C : CUFFT_D2Z, n, batch, real_dist ? real_dist : cells,
                      (cudaStream_t)stream, &h);
    if (st) return st;
    cufftResult r = dtype == CNPC_F32
                        ? cufftExecR2C(h, (cufftReal *)d_real, (cufftComplex *)d_spec)
                        : cufftExecD2Z(h, (cufftDoubleReal *)d_real, (cufftDoubleComplex *)d_spec);
    if (r != CUFFT_SUCCESS) return fail(ctx, CNPC_ECUFFT, "cufftExec r2c failed " + std::to_string((int)r));
    return CNPC_OK;
}

int cnpc_fft_c2r(cnpc_ctx *ctx, int dtype, int n, int batch, void *d_spec, void *d_real, int64_t real_dist,
                 cnpc_stream_t stream) {
    CNPC_REQUIRE(ctx, n >= 2 && n % 2 == 0 && n <= 2048, "n must be even, 2..2048");
    CNPC_REQUIRE(ctx, batch >= 1, "batch must be >= 1");
    CNPC_REQUIRE(ctx, d_real && d_spec, "null buffer");
    CNPC_REQUIRE(ctx, dtype == CNPC_F32 || dtype == CNPC_F64, "bad dtype");
    cufftHandle h;
    const long long cells = (long long)n * n * n;
    CNPC_REQUIRE(ctx, real_dist == 0 || real_dist >= cells, "real_dist must be 0 or >= n^3");
    CNPC_REQUIRE(ctx, real_dist < (1ll << 31), "real_dist too large");
    int st = get_plan(ctx, dtype == CNPC_F32 ? CUFFT_C2R : CUFFT_Z2D, n, batch, real_dist ? real_dist : cells,
                      (cudaStream_t)stream, &h);
    if (st) return st;
    cufftResult r = dtype == CNPC_F32
                        ? cufftExecC2R(h, (cufftComplex *)d_spec, (cufftReal *)d_real)
                        : cufftExecZ2D(h, (cufftDoubleComplex *)d_spec, (cufftDoubleReal *)d_real);
    if (r != CUFFT_SUCCESS) return fail(ctx, CNPC_ECUFFT, "cufftExec c2r failed " + std::to_string((int)r));
    return CNPC_OK;
}

}  // extern "C"
