// GEMM precision dispatch and the not-yet-specialised entry points.
#include <cuda_runtime.h>

#include "internal.h"
#include "tuner.h"

namespace chai {

int launch_gemm_simt(chai_cuda_ctx* ctx, const chai_gemm_desc* d);
int launch_gemm_tc(chai_cuda_ctx* ctx, const chai_gemm_desc* d, int precision);

int launch_gemm(chai_cuda_ctx* ctx, const chai_gemm_desc* d)
{
    int p = d->precision == CHAI_GEMM_AUTO ? ctx->cfg.gemm_precision : d->precision;
    if (d->m < 0 || d->n < 0 || d->k < 0) return set_error(ctx, CHAI_ERR_INVALID, "gemm: negative size");
    switch (p) {
        case CHAI_GEMM_FP32:
        case CHAI_GEMM_FP64:
            return launch_gemm_simt(ctx, d);
        case CHAI_GEMM_TF32:
        case CHAI_GEMM_BF16:
        case CHAI_GEMM_BF16X3:
        case CHAI_GEMM_BF16X6:
        case CHAI_GEMM_FP8:
            return launch_gemm_tc(ctx, d, p);
    }
    return set_error(ctx, CHAI_ERR_INVALID, "gemm: unknown precision");
}

}  // namespace chai
