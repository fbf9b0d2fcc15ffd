// GEMM / GEMV tile-configuration tuner (replaces autotune/StandardEM.cpp,
// autotune/AutoTuneEM.cpp, autotune/AutoTuneBench.cpp and the journal of
// autotune/AutoTuneMemo.hpp).  See tuner.cpp.
#pragma once

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "chai_b200.h"

struct chai_cuda_ctx;

namespace chai {

// tcgen05 GEMM tile configuration (gemm_tc.cu): M-tile height (128: one CTA
// per tile; 256: a CTA pair on two SMs, cta_group::2), N-tile width (one-CTA
// tiles), pipeline stages, tile-raster group height.
struct TcCfg {
    int bm = 256, bn = 256, stages = 4, group_m = 16;
};
// The configuration of an untuned shape: 256 x 256 CTA-pair tiles, unless
// they would keep fewer than half of the `sms` SMs busy (small products, e.g.
// 512^2: 4 pairs on 8 SMs); then one-CTA 128 x 64 tiles, 8x as many (128 x
// 128 or 128 x 256 tiles would still leave over half of the SMs idle there).
inline TcCfg default_tc_cfg(long long m, long long n, int sms)
{
    TcCfg c;
    const long long pairs = ((m + 255) / 256) * ((n + 255) / 256);
    if (2 * pairs >= sms / 2) return c;
    c.bm = 128;
    c.bn = 64;
    return c;
}
bool tuned_tc_cfg(chai_cuda_ctx* ctx, long long m, long long n, long long k, int precision, TcCfg* out);

// GEMV configuration (gemv.cu): warps (rows) per block, 16-byte loads in
// flight per lane.
// warps = 0 selects the bulk-copy kernel (A streamed through shared memory by
// cp.async.bulk) when the operands are 16-byte aligned.
struct GemvCfg {
    int warps = 0, unroll = 1;
};
bool tuned_gemv_cfg(chai_cuda_ctx* ctx, long long m, long long n, int prec, GemvCfg* out);

// b_planes: B already split by gemm_split_b (one problem, not fp8), or null
int launch_gemm_tc_cfg(chai_cuda_ctx* ctx, const chai_gemm_desc* d, int precision, const TcCfg* cfg,
                       const void* b_planes = nullptr);
size_t gemm_b_planes_bytes(int precision, long long k, long long n);
int gemm_split_b(chai_cuda_ctx* ctx, int precision, const float* b, long long ldb, long long k, long long n,
                 void* out);
int launch_gemv_cfg(chai_cuda_ctx* ctx, uint32_t prec, int trans, int64_t m, int64_t n, double alpha, const void* a,
                    int64_t lda, const void* x, double beta, void* y, const GemvCfg* cfg);

void preload_gemm_kernels();
void preload_gemv_kernels();

// The cost model: features (tuner.cpp) -> 3 x 128 ReLU -> log runtime (mlp.cu).
constexpr int MLP_IN = 14, MLP_H = 128;
class Mlp;

class Tuner {
public:
    explicit Tuner(chai_cuda_ctx* ctx);
    ~Tuner();
    int tune(const chai_gemm_key* key, int mode, chai_gemm_cfg* out);
    int sweep(const chai_gemm_key* key, chai_gemm_cfg* out, int cap, int* n);
    int load(const std::string& path);
    int save(const std::string& path) const;
    bool lookup(const chai_gemm_key* key, chai_gemm_cfg* out) const;
    Mlp* mlp() { return mlp_; }
    static std::vector<chai_gemm_cfg> space(const chai_gemm_key& key);
    static void features(const chai_gemm_key& key, const chai_gemm_cfg& cfg, float* f);
    int top_k = 3;

private:
    chai_cuda_ctx* ctx_;
    Mlp* mlp_;
    std::map<std::tuple<long long, long long, long long, int, int>, chai_gemm_cfg> db_;
    std::map<std::string, int> bad_;     // configurations that crashed (journal)
    std::string journal_;
    void* bufs_[3] = {nullptr, nullptr, nullptr};
    size_t buf_bytes_[3] = {0, 0, 0};
    bool preloaded_ = false;
    int time_cfg(const chai_gemm_key& key, chai_gemm_cfg& cfg, int reps, bool warm);
    int ensure_operands(const chai_gemm_key& key);
};

}  // namespace chai
