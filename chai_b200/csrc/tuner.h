// GEMM / GEMV tile-configuration tuner (replaces autotune/StandardEM.cpp,
// autotune/AutoTuneEM.cpp, autotune/AutoTuneBench.cpp and the journal of
// autotune/AutoTuneMemo.hpp).  See tuner.cpp.
#pragma once

#include <map>
#include <string>
#include <tuple>

#include "chai_b200.h"

struct chai_cuda_ctx;

namespace chai {

class Tuner {
public:
    explicit Tuner(chai_cuda_ctx* ctx) : ctx_(ctx) {}
    int tune(const chai_gemm_key* key, int mode, chai_gemm_cfg* out);
    int load(const std::string& path);
    int save(const std::string& path) const;
    // configuration to use for a GEMM without tuning (tuned entry if any)
    bool lookup(const chai_gemm_key* key, chai_gemm_cfg* out) const;

private:
    chai_cuda_ctx* ctx_;
    std::map<std::tuple<long long, long long, long long, int, int>, chai_gemm_cfg> db_;
};

}  // namespace chai
