// NVRTC compilation and driver-API launch of specialised trace kernels.
#include "jit.h"

#include <cuda.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <vector>

#include "internal.h"

namespace chai {

uint64_t fnv1a64(const void* data, size_t n, uint64_t h)
{
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; i++) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

typedef CUresult (*PFN_load)(CUmodule*, const void*);
typedef CUresult (*PFN_getfn)(CUfunction*, CUmodule, const char*);
typedef CUresult (*PFN_launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               CUstream, void**, void**);
typedef CUresult (*PFN_unload)(CUmodule);
typedef CUresult (*PFN_setattr)(CUfunction, CUfunction_attribute, int);

Jit::Jit(chai_cuda_ctx* ctx) : ctx_(ctx) {}

Jit::~Jit()
{
    if (p_unload_)
        for (auto& kv : modules_) reinterpret_cast<PFN_unload>(p_unload_)((CUmodule)kv.second);
}

int Jit::resolve()
{
    if (p_launch_) return CHAI_OK;
    struct { const char* name; void** slot; } syms[] = {
        {"cuModuleLoadData", &p_load_}, {"cuModuleGetFunction", &p_getfn_}, {"cuLaunchKernel", &p_launch_},
        {"cuModuleUnload", &p_unload_}, {"cuFuncSetAttribute", &p_setattr_}};
    for (auto& s : syms) {
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPointByVersion(s.name, s.slot, 12000, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !*s.slot)
            return set_error(ctx_, CHAI_ERR_NO_DEVICE, std::string("driver entry point missing: ") + s.name);
    }
    return CHAI_OK;
}

static std::string cache_path(const std::string& dir, uint64_t h, uint64_t h2)
{
    char buf[48];
    snprintf(buf, sizeof buf, "%016llx%016llx", (unsigned long long)h, (unsigned long long)h2);
    return dir + "/chai_" + buf + ".cubin";
}

// NVRTC options of every trace kernel.  --fmad=false: every traced operation
// rounds on its own, as the reference interpreter's scalar functors do (no
// multiply-add contraction).
static const char* const kNvrtcOpts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "-lineinfo",
                                         "--fmad=false"};
static const int kNvrtcNopts = (int)(sizeof kNvrtcOpts / sizeof kNvrtcOpts[0]);

// What a compiled kernel depends on besides its source: the NVRTC version and
// the options.  It seeds the on-disk cache key, so cubins built by another
// NVRTC or with other options are never loaded.
static uint64_t build_identity()
{
    int major = 0, minor = 0;
    nvrtcVersion(&major, &minor);
    std::string id = "nvrtc " + std::to_string(major) + "." + std::to_string(minor);
    for (int i = 0; i < kNvrtcNopts; i++) (id += ' ') += kNvrtcOpts[i];
    return fnv1a64(id.data(), id.size());
}

int Jit::get(const std::string& body, const char* name, void** fn)
{
    int st = compile_only_ ? CHAI_OK : resolve();
    if (st) return st;
    // the prelude is fixed for the life of the library: the in-memory key is
    // the kernel name and the whole body (compared in full, not by hash)
    std::string key(name);
    key += '\0';
    key += body;
    std::lock_guard<std::mutex> g(mu_);
    auto it = functions_.find(key);
    if (it != functions_.end()) {
        *fn = it->second;
        return CHAI_OK;
    }
    std::string src;
    src.reserve(body.size() + 32768);
    src += kChaiRngSrc;
    src += "\n";
    src += kChaiOpsSrc;
    src += "\n";
    src += kChaiTracePreludeSrc;
    src += "\n";
    src += body;
    // on-disk cache entries are keyed by the NVRTC version and options and the
    // whole source (prelude included), under two independent 64-bit hashes
    static const uint64_t ident = build_identity();
    const uint64_t hdisk = fnv1a64(name, strlen(name), fnv1a64(src.data(), src.size(), ident));
    const uint64_t hdisk2 = fnv1a64(src.data(), src.size(), fnv1a64(name, strlen(name), ident ^ 0x9E3779B97F4A7C15ull));
    std::vector<char> cubin;
    const char* dir = compile_only_ ? nullptr : ctx_->cfg.jit_cache.empty() ? getenv("CHAI_JIT_CACHE") : ctx_->cfg.jit_cache.c_str();
    if (dir && *dir) {
        std::ifstream f(cache_path(dir, hdisk, hdisk2), std::ios::binary);
        if (f) cubin.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    if (cubin.empty()) {
        nvrtcProgram prog;
        if (nvrtcCreateProgram(&prog, src.c_str(), "chai_trace.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
            return set_error(ctx_, CHAI_ERR_JIT, "nvrtcCreateProgram failed");
        nvrtcResult r = nvrtcCompileProgram(prog, kNvrtcNopts, kNvrtcOpts);
        if (r != NVRTC_SUCCESS) {
            size_t n = 0;
            nvrtcGetProgramLogSize(prog, &n);
            std::string log(n, '\0');
            nvrtcGetProgramLog(prog, &log[0]);
            nvrtcDestroyProgram(&prog);
            return set_error(ctx_, CHAI_ERR_JIT, "nvrtc: " + log.substr(0, 4000));
        }
        size_t n = 0;
        nvrtcGetCUBINSize(prog, &n);
        cubin.resize(n);
        nvrtcGetCUBIN(prog, cubin.data());
        nvrtcDestroyProgram(&prog);
        compiles_++;
        if (compile_only_) {
            *fn = nullptr;
            return CHAI_OK;
        }
        if (dir && *dir) {
            // write to a private name, then rename: a reader never sees a partial file
            const std::string final_path = cache_path(dir, hdisk, hdisk2);
            const std::string tmp = final_path + ".tmp" + std::to_string((unsigned long long)(uintptr_t)this);
            {
                std::ofstream f(tmp, std::ios::binary);
                if (f) f.write(cubin.data(), (std::streamsize)cubin.size());
            }
            std::rename(tmp.c_str(), final_path.c_str());
        }
    }
    CUmodule mod;
    CUresult cr = reinterpret_cast<PFN_load>(p_load_)(&mod, cubin.data());
    if (cr != CUDA_SUCCESS) return set_error(ctx_, CHAI_ERR_JIT, "cuModuleLoadData failed");
    CUfunction f;
    cr = reinterpret_cast<PFN_getfn>(p_getfn_)(&f, mod, name);
    if (cr != CUDA_SUCCESS) return set_error(ctx_, CHAI_ERR_JIT, std::string("kernel not found: ") + name);
    modules_[key] = mod;
    functions_[key] = f;
    *fn = f;
    return CHAI_OK;
}

int Jit::launch(void* fn, dim3 grid, dim3 block, size_t smem, void** args)
{
    if (smem > 48 * 1024)
        reinterpret_cast<PFN_setattr>(p_setattr_)((CUfunction)fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                                  (int)smem);
    CUresult r = reinterpret_cast<PFN_launch>(p_launch_)((CUfunction)fn, grid.x, grid.y, grid.z, block.x, block.y,
                                                         block.z, (unsigned)smem, (CUstream)ctx_->stream, args,
                                                         nullptr);
    if (r != CUDA_SUCCESS) return set_error(ctx_, CHAI_ERR_LAUNCH, "cuLaunchKernel failed");
    return CHAI_OK;
}

}  // namespace chai
