// GEMM precision dispatch and the not-yet-specialised entry points.
#include <cuda_runtime.h>

#include "internal.h"
#include "tuner.h"

namespace chai {

int launch_gemm_simt(chai_cuda_ctx* ctx, const chai_gemm_desc* d);
int launch_gemm_tc(chai_cuda_ctx* ctx, const chai_gemm_desc* d, int precision);

// The arithmetic of an f32 matmul whose precision is CHAI_GEMM_AUTO.  With
// GemmPrecision=auto (the default) every f32 product with M, N >= 32 and
// K >= 16 runs on the tcgen05 tensor cores as the bf16x3 split-precision GEMM
// (FP32-level error, three bf16 products); thinner products -- matrix-vector
// shapes the 128-row tensor-core tiles would mostly pad -- run on the FP32
// CUDA-core kernel.  The reference routes every matmul statement to its one
// auto-tuned GEMM (jitstmt/MakeStmt.cpp:374-463); a configured
// GemmPrecision=<name> fixes the arithmetic instead.
int resolve_precision(chai_cuda_ctx* ctx, int precision, long long m, long long n, long long k)
{
    if (precision != CHAI_GEMM_AUTO) return precision;
    if (ctx->cfg.gemm_precision != CHAI_GEMM_AUTO) return ctx->cfg.gemm_precision;
    return (m >= 32 && n >= 32 && k >= 16) ? CHAI_GEMM_BF16X3 : CHAI_GEMM_FP32;
}

int launch_gemm(chai_cuda_ctx* ctx, const chai_gemm_desc* d)
{
    int p = resolve_precision(ctx, d->precision, d->m, d->n, d->k);
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
