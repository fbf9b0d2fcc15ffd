// Entry points whose specialised kernels live in later files of this build.
#include "internal.h"
#include "tuner.h"

namespace chai {

int Tuner::tune(const chai_gemm_key* key, int mode, chai_gemm_cfg* out)
{
    (void)key; (void)mode; (void)out;
    return CHAI_ERR_UNSUPPORTED;
}
int Tuner::load(const std::string& path) { (void)path; return CHAI_OK; }
int Tuner::save(const std::string& path) const { (void)path; return CHAI_OK; }
bool Tuner::lookup(const chai_gemm_key* key, chai_gemm_cfg* out) const { (void)key; (void)out; return false; }

}  // namespace chai

using namespace chai;

extern "C" {

int chai_cuda_tune(chai_cuda_ctx* ctx, const chai_gemm_key* key, int mode, chai_gemm_cfg* out)
{
    if (!ctx || !key || !out) return CHAI_ERR_INVALID;
    return ctx->tuner->tune(key, mode, out);
}

int chai_cuda_tune_db_load(chai_cuda_ctx* ctx, const char* path)
{
    if (!ctx || !path) return CHAI_ERR_INVALID;
    return ctx->tuner->load(path);
}

int chai_cuda_tune_db_save(chai_cuda_ctx* ctx, const char* path)
{
    if (!ctx || !path) return CHAI_ERR_INVALID;
    return ctx->tuner->save(path);
}

}  // extern "C"
