// Runtime specialisation of trace kernels.  A trace's fused element kernel is
// a hand-written template (chai_trace_prelude) instantiated with the trace's
// expression body; it is compiled once per distinct body for sm_100a with
// NVRTC and cached in memory (keyed by the whole generated source) and
// optionally on disk (keyed by two 64-bit hashes of the source, the NVRTC
// version and the options), the way the reference caches OpenCL kernels by
// trace hash (kernel/KernelCache.cpp:21-119) -- but the key covers every byte
// of the generated source, so traces that differ only in a literal never share
// a kernel (bytecode/HashBC.cpp:44-50 truncates literals to integers).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>

struct chai_cuda_ctx;

namespace chai {

uint64_t fnv1a64(const void* data, size_t n, uint64_t h = 1469598103934665603ull);

class Jit {
public:
    explicit Jit(chai_cuda_ctx* ctx);
    ~Jit();
    // Compile `src` (prelude prepended) if not cached and return the kernel
    // `name`.  Returns a chai_status.
    int get(const std::string& body, const char* name, void** fn);
    int launch(void* fn, dim3 grid, dim3 block, size_t smem, void** args);
    size_t compiles() const { return compiles_; }
    // compile with NVRTC but load nothing (no device needed)
    void set_compile_only(bool v) { compile_only_ = v; }

private:
    chai_cuda_ctx* ctx_;
    std::mutex mu_;
    std::map<std::string, void*> modules_;     // name + body -> CUmodule
    std::map<std::string, void*> functions_;   // name + body -> CUfunction
    size_t compiles_ = 0;
    bool compile_only_ = false;
    // driver entry points resolved through the runtime (no libcuda link)
    void* p_load_ = nullptr;
    void* p_getfn_ = nullptr;
    void* p_launch_ = nullptr;
    void* p_unload_ = nullptr;
    void* p_setattr_ = nullptr;
    int resolve();
};

// Embedded device headers (generated at build time from csrc/*.cuh).
extern const char* const kChaiRngSrc;
extern const char* const kChaiOpsSrc;
extern const char* const kChaiTracePreludeSrc;

}  // namespace chai
