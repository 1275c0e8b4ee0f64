// Internal (host-side) declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "cosmonpc_b200.h"

struct cnpc_ctx {
    int device = 0;
    std::string last_error;
    // cuFFT plans keyed by (type, n, batch, real-field distance), each with the
    // work-area size it needs; the plans share one work area (fft_ws), set before
    // every execution, so cached plans of several batch depths and precisions
    // do not each hold a workspace of their own
    struct FftPlan {
        cufftHandle h;
        size_t work;
    };
    std::map<std::tuple<int, int, int, long long>, FftPlan> plans;
    void *fft_ws = nullptr;
    size_t fft_ws_bytes = 0;
    // scratch for per-block partial sums of the x-space reductions
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    // workspace of the tiled paint (tile counts, offsets, sorted particles)
    void *paint_ws = nullptr;
    size_t paint_ws_bytes = 0;
    // workspace of the catalog and survey reductions (block counts, partials)
    void *aux = nullptr;
    size_t aux_bytes = 0;
    // workspace of the fused shell-field transform (output table + pass-1 columns)
    void *shell_ws = nullptr;
    size_t shell_ws_bytes = 0;
    int num_sms = 148;
    // status word of the bounded device waits (CNPC_OK or CNPC_ETIMEOUT),
    // sticky until cnpc_ctx_take_status reads and clears it
    int *d_status = nullptr;
    // polls of a bounded mbarrier wait before it gives up
    long long wait_limit = 1ll << 22;
};

namespace cnpc {

int fail(cnpc_ctx *ctx, int status, const std::string &msg);
int check_cuda(cnpc_ctx *ctx, cudaError_t e, const char *what);
int check_launch(cnpc_ctx *ctx, const char *what);
int ensure_scratch(cnpc_ctx *ctx, size_t bytes, cudaStream_t stream);
int ensure_buffer(cnpc_ctx *ctx, void **buf, size_t *have, size_t bytes, cudaStream_t stream);
int ensure_status(cnpc_ctx *ctx);

}  // namespace cnpc

#define CNPC_REQUIRE(ctx, cond, msg)                                  \
    do {                                                              \
        if (!(cond)) return ::cnpc::fail((ctx), CNPC_EINVAL, (msg));  \
    } while (0)

#define CNPC_GUARD_BEGIN try {
#define CNPC_GUARD_END(ctx)                                                       \
    }                                                                             \
    catch (const std::exception &ex) {                                            \
        return ::cnpc::fail((ctx), CNPC_EINVAL, std::string("exception: ") + ex.what()); \
    }                                                                             \
    catch (...) {                                                                 \
        return ::cnpc::fail((ctx), CNPC_EINVAL, "unknown exception");             \
    }
