// Context life cycle and device memory: the C-ABI half that replaces
// Translator::initDevice (runtime/Translator.cpp:353-364) and the JIT memory
// manager MemTrans (memmgr/MemTrans.hpp:31-235: memalloc, swizzle,
// untrackMem).  Device arrays stay resident in HBM between traces; only
// explicit uploads (make1/make2 data) and readbacks (read_scalar/read1/read2)
// cross PCIe/C2C.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "internal.h"
#include "jit.h"
#include "tuner.h"

namespace chai {

void many_release(chai_cuda_ctx* ctx);

int set_error(chai_cuda_ctx* ctx, int status, const std::string& msg)
{
    if (ctx) {
        std::lock_guard<std::mutex> g(ctx->err_mutex);
        ctx->last_error = msg;
    }
    return status;
}

int cuda_status(chai_cuda_ctx* ctx, cudaError_t e, const char* what)
{
    int st = CHAI_ERR_LAUNCH;
    if (e == cudaErrorMemoryAllocation) st = CHAI_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) st = CHAI_ERR_NO_DEVICE;
    std::ostringstream os;
    os << what << ": " << cudaGetErrorString(e);
    return set_error(ctx, st, os.str());
}

size_t prec_bytes(uint32_t prec)
{
    switch (prec) {
        case CHAI_U32: case CHAI_I32: case CHAI_F32: return 4;
        case CHAI_F64: return 8;
    }
    return 0;
}

// Host-side fault injection: CHAI_FAULT_INJECT=<site>[,<site>...] makes the
// named entry point fail with CHAI_ERR_INJECTED before touching the GPU, so
// the caller's fall-back path (DEVICE_FAILURE -> another device) can be
// exercised without faulting a GPU.
bool fault_injected(const char* site)
{
    const char* env = getenv("CHAI_FAULT_INJECT");
    if (!env || !*env) return false;
    std::string s(env), want(site);
    size_t pos = 0;
    while (pos <= s.size()) {
        size_t end = s.find(',', pos);
        if (end == std::string::npos) end = s.size();
        if (s.compare(pos, end - pos, want) == 0 || s.compare(pos, end - pos, "all") == 0) return true;
        pos = end + 1;
    }
    return false;
}

void ktime_begin(chai_cuda_ctx* ctx, const char* name, cudaEvent_t* ev)
{
    (void)name;
    ev[0] = ev[1] = nullptr;
    if (!ctx->kernel_timing || ctx->capturing) return;
    for (int k = 0; k < 2; k++) {
        if (!ctx->event_pool.empty()) {
            ev[k] = ctx->event_pool.back();
            ctx->event_pool.pop_back();
        } else {
            cudaEventCreate(&ev[k]);
        }
    }
    cudaEventRecord(ev[0], ctx->stream);
}

void ktime_end(chai_cuda_ctx* ctx, const char* name, cudaEvent_t* ev)
{
    if (!ctx->kernel_timing || !ev[0]) return;
    cudaEventRecord(ev[1], ctx->stream);
    ctx->kstats[name].pending.push_back(std::make_pair(ev[0], ev[1]));
}

Buffer* find_buffer(chai_cuda_ctx* ctx, uint64_t id)
{
    std::lock_guard<std::mutex> g(ctx->mem_mutex);
    auto it = ctx->buffers.find(id);
    return it == ctx->buffers.end() ? nullptr : &it->second;
}

int alloc_buffer(chai_cuda_ctx* ctx, uint64_t id, size_t bytes)
{
    if (fault_injected("alloc")) return set_error(ctx, CHAI_ERR_INJECTED, "injected allocation failure");
    {
        std::lock_guard<std::mutex> g(ctx->mem_mutex);
        auto it = ctx->buffers.find(id);
        if (it != ctx->buffers.end()) {
            if (it->second.bytes >= bytes) return CHAI_OK;
            if (!it->second.owned) return set_error(ctx, CHAI_ERR_INVALID, "wrapped buffer too small");
        }
    }
    void* p = nullptr;
    const size_t rounded = (bytes + 255) & ~size_t(255);
    cudaError_t e = cudaMallocAsync(&p, rounded ? rounded : 256, ctx->stream);
    if (e != cudaSuccess) return cuda_status(ctx, e, "cudaMallocAsync");
    std::lock_guard<std::mutex> g(ctx->mem_mutex);
    auto it = ctx->buffers.find(id);
    if (it != ctx->buffers.end()) cudaFreeAsync(it->second.ptr, ctx->stream);
    ctx->buffers[id] = Buffer{p, bytes, true};
    return CHAI_OK;
}

int ensure_scratch(chai_cuda_ctx* ctx, size_t bytes)
{
    if (ctx->scratch_bytes >= bytes) return CHAI_OK;
    // a graph must not own the context scratch: growing it ends the capture
    if (ctx->capturing) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "scratch growth during graph capture");
    const size_t want = bytes < (64u << 20) ? (64u << 20) : (bytes + (bytes >> 2));
    if (ctx->scratch) CHAI_CUDA_TRY(ctx, cudaFreeAsync(ctx->scratch, ctx->stream));
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    CHAI_CUDA_TRY(ctx, cudaMallocAsync(&ctx->scratch, want, ctx->stream));
    ctx->scratch_bytes = want;
    return CHAI_OK;
}

void parse_config(chai::Config& c, const char* text)
{
    if (!text) return;
    std::istringstream is(text);
    std::string tok;
    while (is >> tok) {
        const size_t eq = tok.find('=');
        if (eq == std::string::npos) continue;   // devspec.cfg keywords without values
        const std::string k = tok.substr(0, eq), v = tok.substr(eq + 1);
        if (k == "GemmPrecision") {
            if (v == "auto") c.gemm_precision = CHAI_GEMM_AUTO;
            else if (v == "fp32") c.gemm_precision = CHAI_GEMM_FP32;
            else if (v == "tf32") c.gemm_precision = CHAI_GEMM_TF32;
            else if (v == "bf16") c.gemm_precision = CHAI_GEMM_BF16;
            else if (v == "bf16x3") c.gemm_precision = CHAI_GEMM_BF16X3;
            else if (v == "bf16x6") c.gemm_precision = CHAI_GEMM_BF16X6;
            else if (v == "fp8") c.gemm_precision = CHAI_GEMM_FP8;
        } else if (k == "RngPi") {
            c.rng_pi = atof(v.c_str());
        } else if (k == "RngLayout") {
            c.rng_layout = (v == "counter") ? 1 : 0;
        } else if (k == "TunerMode") {
            c.tuner_mode = (v == "exhaustive") ? CHAI_TUNE_EXHAUSTIVE : CHAI_TUNE_LEARNED;
        } else if (k == "TopK") {
            c.top_k = std::max(1, atoi(v.c_str()));
        } else if (k == "StencilRows") {
            c.stencil_rows = atoi(v.c_str());
        } else if (k == "FuseMaxAffine") {
            c.fuse_max_affine = v != "0" && v != "off";
        } else if (k == "ReduceAccum") {
            c.reduce_accum_f32 = v == "f32";
        } else if (k == "StencilRowsPerThread") {
            c.stencil_rows_per_thread = std::max(1, std::min(4, atoi(v.c_str())));
        } else if (k == "StencilMinBlocks") {
            c.stencil_min_blocks = std::max(0, std::min(8, atoi(v.c_str())));
        } else if (k == "GemmPair") {
            c.gemm_pair = v != "0" && v != "off";
        } else if (k == "GemmPairSeg") {
            c.gemm_pair_seg = std::max(1, atoi(v.c_str()));
        } else if (k == "GemmSplitK") {
            c.gemm_split_k = v != "0" && v != "off";
        } else if (k == "GemmStages") {
            c.gemm_stages = std::max(0, atoi(v.c_str()));
        } else if (k == "GroupedPair") {
            c.grouped_pair = v != "0" && v != "off";
        } else if (k == "GroupedTmaB") {
            c.grouped_tma_b = v != "0" && v != "off";
        } else if (k == "GroupedExact") {
            c.grouped_exact = v != "0" && v != "off";
        } else if (k == "GroupedSplit") {
            c.grouped_fused = v != "prepass";
        } else if (k == "PackF32") {
            c.pack_f32 = v != "0" && v != "off";
        } else if (k == "PackF32Stencil") {
            c.pack_f32_stencil = v != "0" && v != "off";
        } else if (k == "StencilBorderTma") {
            c.stencil_border_tma = v != "0" && v != "off";
        } else if (k == "PlanCache") {
            c.plan_cache = v != "0" && v != "off";
        } else if (k == "PlanGraph") {
            c.plan_graph = (v == "auto") ? -1 : (v != "0" && v != "off") ? 1 : 0;
        } else if (k == "TuneJournal") {
            c.tune_journal = v;
        } else if (k == "TuneDB") {
            c.tune_db = v;
        } else if (k == "JitCache") {
            c.jit_cache = v;
        }
    }
}

}  // namespace chai

using namespace chai;

extern "C" {

const char* chai_cuda_error_string(int status)
{
    switch (status) {
        case CHAI_OK: return "ok";
        case CHAI_ERR_INVALID: return "invalid argument or malformed trace";
        case CHAI_ERR_UNSUPPORTED: return "unsupported operation";
        case CHAI_ERR_OOM: return "device out of memory";
        case CHAI_ERR_LAUNCH: return "kernel launch or execution failed";
        case CHAI_ERR_TIMEOUT: return "bounded device wait gave up";
        case CHAI_ERR_NOT_FOUND: return "unknown buffer id";
        case CHAI_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
        case CHAI_ERR_JIT: return "runtime compilation failed";
        case CHAI_ERR_INJECTED: return "injected failure";
    }
    return "unknown status";
}

int chai_cuda_init(int device, const char* config, chai_cuda_ctx** out)
{
    if (!out) return CHAI_ERR_INVALID;
    *out = nullptr;
    if (fault_injected("init")) return CHAI_ERR_INJECTED;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0 || device < 0 || device >= count) {
        cudaGetLastError();
        return CHAI_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return CHAI_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return CHAI_ERR_NO_DEVICE;
    auto* ctx = new chai_cuda_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    parse_config(ctx->cfg, config);
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return CHAI_ERR_NO_DEVICE;
    }
    ctx->stream = ctx->own_stream;
    if (cudaMallocHost(&ctx->pinned, 4096 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&ctx->status_word, 64) != cudaSuccess ||
        cudaMemset(ctx->status_word, 0, 64) != cudaSuccess) {
        chai_cuda_shutdown(ctx);
        return CHAI_ERR_OOM;
    }
    ctx->pinned_count = 4096;
    ctx->kernel_timing = getenv("CHAI_KERNEL_TIMING") && atoi(getenv("CHAI_KERNEL_TIMING")) != 0;
    ctx->jit.reset(new Jit(ctx));
    ctx->tuner.reset(new Tuner(ctx));
    if (!ctx->cfg.tune_db.empty() || !ctx->cfg.tune_journal.empty()) ctx->tuner->load(ctx->cfg.tune_db);
    *out = ctx;
    return CHAI_OK;
}

int chai_cuda_shutdown(chai_cuda_ctx* ctx)
{
    if (!ctx) return CHAI_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    many_release(ctx);
    host_gemm_release(ctx);
    for (auto& kv : ctx->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    ctx->graphs.clear();
    ctx->tuner.reset();
    ctx->jit.reset();
    for (auto& kv : ctx->kstats)
        for (auto& p : kv.second.pending) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    for (auto& kv : ctx->buffers)
        if (kv.second.owned && kv.second.ptr) cudaFree(kv.second.ptr);
    ctx->buffers.clear();
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->gplan.dev) cudaFree(ctx->gplan.dev);
    if (ctx->gplan.maps) cudaFree(ctx->gplan.maps);
    if (ctx->status_word) cudaFree(ctx->status_word);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return CHAI_OK;
}

// Device time of the library's hot kernels, recorded with CUDA events on the
// context stream when CHAI_KERNEL_TIMING=1 (the counterpart of the reference's
// per-dispatch timing in Scheduler::_workStat, runtime/Scheduler.cpp:198-220).
int chai_cuda_kernel_stats(chai_cuda_ctx* ctx, const char* name, double* total_ms, uint64_t* launches, int reset)
{
    if (!ctx || !name) return CHAI_ERR_INVALID;
    if (std::string(name) == "plan_replay") {      // evaluations replayed from the plan cache
        if (total_ms) *total_ms = 0;
        if (launches) *launches = ctx->plan_hits;
        if (reset) ctx->plan_hits = 0;
        return CHAI_OK;
    }
    if (std::string(name) == "plan_graph") {       // replays launched from a captured CUDA graph
        if (total_ms) *total_ms = 0;
        if (launches) *launches = ctx->graph_launches;
        if (reset) ctx->graph_launches = 0;
        return CHAI_OK;
    }
    if (std::string(name) == "grouped_fused") {    // grouped GEMMs split inside the GEMM kernel
        if (total_ms) *total_ms = 0;
        if (launches) *launches = ctx->fused_launches;
        if (reset) ctx->fused_launches = 0;
        return CHAI_OK;
    }
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    auto& st = ctx->kstats[name];
    for (auto& p : st.pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.first, p.second);
        st.ms += ms;
        st.launches++;
        ctx->event_pool.push_back(p.first);
        ctx->event_pool.push_back(p.second);
    }
    st.pending.clear();
    if (total_ms) *total_ms = st.ms;
    if (launches) *launches = st.launches;
    if (reset) { st.ms = 0; st.launches = 0; }
    return CHAI_OK;
}

int chai_cuda_selftest_wait(chai_cuda_ctx* ctx, double limit_ms)
{
    if (!ctx || !(limit_ms > 0) || limit_ms > 2000) return CHAI_ERR_INVALID;
    int st = launch_wait_selftest(ctx, limit_ms);
    if (st) return st;
    return chai_cuda_synchronize(ctx);
}

int chai_cuda_synchronize(chai_cuda_ctx* ctx)
{
    if (!ctx) return CHAI_ERR_INVALID;
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    int st = 0;
    CHAI_CUDA_TRY(ctx, cudaMemcpy(&st, ctx->status_word, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) {
        cudaMemset(ctx->status_word, 0, sizeof(int));
        return set_error(ctx, CHAI_ERR_TIMEOUT, "device status word set by a kernel");
    }
    return CHAI_OK;
}

const char* chai_cuda_last_error(chai_cuda_ctx* ctx)
{
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

int chai_cuda_set_stream(chai_cuda_ctx* ctx, void* stream)
{
    if (!ctx) return CHAI_ERR_INVALID;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return CHAI_OK;
}

int chai_cuda_buffer_alloc(chai_cuda_ctx* ctx, uint64_t id, size_t bytes)
{
    if (!ctx) return CHAI_ERR_INVALID;
    std::lock_guard<std::mutex> cap(ctx->capture_mutex);      // not inside another thread's capture
    return alloc_buffer(ctx, id, bytes);
}

int chai_cuda_buffer_wrap(chai_cuda_ctx* ctx, uint64_t id, void* device_ptr, size_t bytes)
{
    if (!ctx || !device_ptr) return CHAI_ERR_INVALID;
    std::lock_guard<std::mutex> g(ctx->mem_mutex);
    auto it = ctx->buffers.find(id);
    if (it != ctx->buffers.end() && it->second.owned) cudaFreeAsync(it->second.ptr, ctx->stream);
    ctx->buffers[id] = Buffer{device_ptr, bytes, false};
    return CHAI_OK;
}

int chai_cuda_buffer_info(chai_cuda_ctx* ctx, uint64_t id, void** device_ptr, size_t* bytes)
{
    if (!ctx) return CHAI_ERR_INVALID;
    Buffer* b = find_buffer(ctx, id);
    if (!b) return set_error(ctx, CHAI_ERR_NOT_FOUND, "buffer_info: unknown id");
    if (device_ptr) *device_ptr = b->ptr;
    if (bytes) *bytes = b->bytes;
    return CHAI_OK;
}

int chai_cuda_upload(chai_cuda_ctx* ctx, uint64_t id, const void* host, size_t bytes)
{
    if (!ctx || (!host && bytes)) return CHAI_ERR_INVALID;
    std::lock_guard<std::mutex> cap(ctx->capture_mutex);      // not inside another thread's capture
    cudaSetDevice(ctx->device);
    int st = alloc_buffer(ctx, id, bytes);
    if (st) return st;
    Buffer* b = find_buffer(ctx, id);
    CHAI_CUDA_TRY(ctx, cudaMemcpyAsync(b->ptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    // pageable sources are staged by the driver; make the call synchronous
    // with respect to the host buffer so the caller may reuse it at once
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return CHAI_OK;
}

int chai_cuda_readback(chai_cuda_ctx* ctx, uint64_t id, void* host, size_t bytes)
{
    if (!ctx || (!host && bytes)) return CHAI_ERR_INVALID;
    std::lock_guard<std::mutex> cap(ctx->capture_mutex);      // not inside another thread's capture
    cudaSetDevice(ctx->device);         // client threads read back too
    Buffer* b = find_buffer(ctx, id);
    if (!b) return set_error(ctx, CHAI_ERR_NOT_FOUND, "readback: unknown id");
    if (bytes > b->bytes) return set_error(ctx, CHAI_ERR_INVALID, "readback larger than buffer");
    CHAI_CUDA_TRY(ctx, cudaMemcpyAsync(host, b->ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return CHAI_OK;
}

int chai_cuda_buffer_copy(chai_cuda_ctx* ctx, uint64_t dst, uint64_t src, size_t bytes)
{
    if (!ctx) return CHAI_ERR_INVALID;
    std::lock_guard<std::mutex> cap(ctx->capture_mutex);      // not inside another thread's capture
    cudaSetDevice(ctx->device);
    Buffer* s = find_buffer(ctx, src);
    if (!s) return set_error(ctx, CHAI_ERR_NOT_FOUND, "buffer_copy: unknown source id");
    if (bytes > s->bytes) return set_error(ctx, CHAI_ERR_INVALID, "buffer_copy larger than the source");
    void* sp = s->ptr;
    int st = alloc_buffer(ctx, dst, bytes);
    if (st) return st;
    Buffer* d = find_buffer(ctx, dst);
    if (bytes) CHAI_CUDA_TRY(ctx, cudaMemcpyAsync(d->ptr, sp, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return CHAI_OK;
}

int chai_cuda_release(chai_cuda_ctx* ctx, uint64_t id)
{
    if (!ctx) return CHAI_ERR_INVALID;
    std::lock_guard<std::mutex> cap(ctx->capture_mutex);      // not inside another thread's capture
    std::lock_guard<std::mutex> g(ctx->mem_mutex);
    auto it = ctx->buffers.find(id);
    if (it == ctx->buffers.end()) return set_error(ctx, CHAI_ERR_NOT_FOUND, "release: unknown id");
    cudaSetDevice(ctx->device);         // client threads release too
    if (it->second.owned) cudaFreeAsync(it->second.ptr, ctx->stream);
    ctx->buffers.erase(it);
    return CHAI_OK;
}

int chai_cuda_rng_fill(chai_cuda_ctx* ctx, const chai_rng_desc* d, void* device_out)
{
    if (!ctx || !d || !device_out) return CHAI_ERR_INVALID;
    return launch_rng_fill(ctx, d, device_out);
}

int chai_cuda_reduce(chai_cuda_ctx* ctx, uint32_t op, uint32_t prec, const void* a, const void* b,
                     uint64_t n, uint32_t slots, double* out)
{
    if (!ctx || !a || !out || op > 2 || (op == 2 && !b) || slots == 0) return CHAI_ERR_INVALID;
    if (slots > ctx->pinned_count) return set_error(ctx, CHAI_ERR_INVALID, "too many slots");
    int st = ensure_scratch(ctx, 0);
    if (st) return st;
    double* dev_out = nullptr;
    CHAI_CUDA_TRY(ctx, cudaMallocAsync(&dev_out, slots * sizeof(double), ctx->stream));
    st = launch_reduce(ctx, op, prec, a, b, n, slots, dev_out);
    if (!st) {
        cudaError_t e = cudaMemcpyAsync(ctx->pinned, dev_out, slots * sizeof(double), cudaMemcpyDeviceToHost,
                                        ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = cuda_status(ctx, e, "reduce readback");
        else memcpy(out, ctx->pinned, slots * sizeof(double));
    }
    cudaFreeAsync(dev_out, ctx->stream);
    return st;
}

int chai_cuda_gemv(chai_cuda_ctx* ctx, uint32_t prec, int trans, int64_t m, int64_t n, double alpha,
                   const void* a, int64_t lda, const void* x, double beta, void* y)
{
    if (!ctx || !a || !x || !y || m < 0 || n < 0) return CHAI_ERR_INVALID;
    return launch_gemv(ctx, prec, trans, m, n, alpha, a, lda, x, beta, y);
}

int chai_cuda_gemm(chai_cuda_ctx* ctx, const chai_gemm_desc* d)
{
    if (!ctx || !d) return CHAI_ERR_INVALID;
    return launch_gemm(ctx, d);
}

int chai_cuda_gemm_grouped(chai_cuda_ctx* ctx, int32_t precision, const chai_gemm_problem* p, int32_t count)
{
    if (!ctx || (!p && count)) return CHAI_ERR_INVALID;
    return launch_gemm_grouped(ctx, precision, p, count);
}

}  // extern "C"
