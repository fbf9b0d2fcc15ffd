// Internal state of a chai_b200 context (host side, C++17).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "chai_b200.h"

namespace chai {

struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool owned = true;
};

struct Config {
    int gemm_precision = CHAI_GEMM_AUTO;     // f32 matmul arithmetic (AUTO: by shape, resolve_precision)
    double rng_pi = 3.14159;                 // M_PI as the reference JIT prints it
    int rng_layout = 0;                      // 0 chai, 1 counter
    int tuner_mode = CHAI_TUNE_LEARNED;
    int top_k = 3;                           // learned tuner: configurations timed
    std::string tune_db;
    std::string tune_journal;                // crash-safe TRY / OK markers of every timing
    bool plan_cache = true;                  // replay recorded plans of repeated traces
    int plan_graph = -1;                     // replay plans from captured CUDA graphs: 1 on, 0 off, -1 unless kernel timing
    int stencil_rows = 0;                    // output rows per stencil tile (multiple of 8, <= 64; 0: 64 or 32 per kernel)
    bool fuse_max_affine = true;             // max of c * s_k - t leaves -> c * max(s_k) - t (exact when t is finite)
    bool reduce_accum_f32 = false;           // f32 reductions: per-thread partials in f32 (block tree, combine FP64)
    int stencil_rows_per_thread = 1;         // output rows per stencil thread (1, 2 or 4; 4 columns each)
    int stencil_min_blocks = 0;              // __launch_bounds__ minimum blocks per SM for stencil kernels (0: none)
    bool grouped_pair = true;                // in-kernel split on 256 x 256 CTA-pair tiles (bf16, bf16x3, K <= 2048)
    bool grouped_tma_b = false;              // in-kernel split: B chunks through TMA (bf16, bf16x3; slower, see gemm_tc.cu)
    bool grouped_exact = true;               // in-kernel split: MMAs cover each tile's N and last K (rounded to 16)
    bool grouped_fused = true;               // grouped GEMM splits f32 operands inside the kernel (else prepass planes)
    bool gemm_pair = true;                   // 256-row GEMM tiles on CTA pairs (cta_group::2) where configured
    int gemm_pair_seg = 64;                  // pair kernel, split precisions: K chunks per promotion segment
    int gemm_stages = 0;                     // GEMM pipeline stages (0: tuned or default)
    bool gemm_split_k = true;                // traced small GEMMs split K over otherwise idle SMs
    bool pack_f32 = true;                    // element kernels issue f32 add / sub as packed f32x2 pairs
    bool pack_f32_stencil = false;           // ... stencil kernels too (slower: re-pairing moves, registers)
    bool stencil_border_tma = true;          // border stencil tiles staged by TMA + wrapped patch loads
    std::string jit_cache;
};

// "Key=value" tokens of an init configuration string into `c` (context.cu)
void parse_config(Config& c, const char* text);

class Jit;      // runtime compilation cache (jit.cpp)
class Tuner;    // learned / exhaustive GEMM tuner (tuner.cpp)
struct Plan;    // recorded device operations of a trace (plan.h)

}  // namespace chai

struct chai_cuda_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex mem_mutex;                                   // buffer table
    std::unordered_map<uint64_t, chai::Buffer> buffers;
    std::mutex err_mutex;
    std::string last_error;
    chai::Config cfg;
    // scratch for reduction partials and split-precision GEMM operands
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    double* pinned = nullptr;                               // pinned host results
    size_t pinned_count = 0;
    int* status_word = nullptr;                             // device error word for bounded waits
    std::unique_ptr<chai::Jit> jit;
    std::unique_ptr<chai::Tuner> tuner;
    uint64_t next_temp_id = 1ull << 62;                     // ids of library-owned temporaries
    // per-kernel device time (CHAI_KERNEL_TIMING=1): name -> events in flight / totals
    bool kernel_timing = false;
    struct KStat { double ms = 0; uint64_t launches = 0; std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending; };
    std::map<std::string, KStat> kstats;
    std::vector<cudaEvent_t> event_pool;
    std::unordered_map<uint64_t, std::shared_ptr<chai::Plan>> plans;   // plan cache, by key hash
    uint64_t plan_hits = 0;
    // captured CUDA graphs of replayed plans: plan key hash -> the device
    // pointers the graph was captured with, and the executable graph
    struct PlanGraph {
        std::vector<void*> sig;              // pointers the instantiated graph was captured with
        cudaGraphExec_t exec = nullptr;
        std::vector<void*> pending;          // pointers of the last plain replay (captured when seen again)
    };
    std::unordered_map<uint64_t, PlanGraph> graphs;
    uint64_t graph_launches = 0;
    bool capturing = false;                                 // a plan replay is being captured
    bool trace_gemm = false;                                // the GEMM being launched is a trace's matmul
    std::mutex capture_mutex;                               // no client-thread stream work during a capture
    // grouped GEMM with the in-kernel split: the device tile records of the
    // last call, reused while the problem array repeats
    struct GroupedPlan {
        std::vector<chai_gemm_problem> problems;
        int S = 0;
        void* dev = nullptr;         // tile records
        size_t bytes = 0;
        long long tiles = 0;
        bool acc2 = false;
        void* maps = nullptr;        // per-problem B tensor maps (B through TMA)
        size_t map_bytes = 0;
        bool bt = false;             // maps valid for `problems`
        bool pair = false;           // tile records of 256 x 256 CTA-pair tiles
    } gplan;
    uint64_t fused_launches = 0;
};

namespace chai {

int set_error(chai_cuda_ctx* ctx, int status, const std::string& msg);
int cuda_status(chai_cuda_ctx* ctx, cudaError_t e, const char* what);
int launch_wait_selftest(chai_cuda_ctx* ctx, double limit_ms);   // gemm_tc.cu

// Grow the context scratch to at least `bytes` (stream-ordered).
int ensure_scratch(chai_cuda_ctx* ctx, size_t bytes);
Buffer* find_buffer(chai_cuda_ctx* ctx, uint64_t id);
int alloc_buffer(chai_cuda_ctx* ctx, uint64_t id, size_t bytes);
bool fault_injected(const char* site);
// bracket a kernel launch with events when kernel timing is on
void ktime_begin(chai_cuda_ctx* ctx, const char* name, cudaEvent_t* ev);
void ktime_end(chai_cuda_ctx* ctx, const char* name, cudaEvent_t* ev);

size_t prec_bytes(uint32_t prec);

// kernels with host launchers (each .cu file)
int launch_rng_fill(chai_cuda_ctx* ctx, const chai_rng_desc* d, void* out);
int launch_reduce(chai_cuda_ctx* ctx, uint32_t op, uint32_t prec, const void* a, const void* b, uint64_t n,
                  uint32_t slots, double* dev_out);
int launch_gemv(chai_cuda_ctx* ctx, uint32_t prec, int trans, int64_t m, int64_t n, double alpha,
                const void* a, int64_t lda, const void* x, double beta, void* y);
int launch_gemm(chai_cuda_ctx* ctx, const chai_gemm_desc* d);
// arithmetic of a CHAI_GEMM_AUTO f32 product of this shape (dispatch.cpp)
int resolve_precision(chai_cuda_ctx* ctx, int precision, long long m, long long n, long long k);
void host_gemm_release(chai_cuda_ctx* ctx);
int launch_gemm_grouped(chai_cuda_ctx* ctx, int32_t precision, const chai_gemm_problem* p, int32_t count);

}  // namespace chai

#define CHAI_CUDA_TRY(ctx, expr)                                              \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) return chai::cuda_status((ctx), _e, #expr);    \
    } while (0)
