/* chai_b200 -- C ABI of the B200 back end for chai traced array programs.
 *
 * This library replaces the reference's OpenCL "Translator" device: the code
 * that turns a recorded trace (a VectorTrace of bytecode stacks) into kernels
 * and runs them, together with the device memory manager and the GEMM
 * autotuner it calls.  The host side that records traces (api/, bytecode/,
 * common/, runtime/ Scheduler) stays the reference's; it reaches this library
 * through a DeviceBase subclass whose sub_evaluate flattens the VectorTrace
 * into a chai_trace_desc and calls chai_cuda_evaluate.
 *
 * Conventions
 *   - Every entry point returns an int status: 0 (CHAI_OK) or a negative
 *     chai_status code.  No C++ exception crosses this boundary.  A non-zero
 *     status maps to DeviceBase::evaluate() == false, which the reference's
 *     scheduler turns into DEVICE_FAILURE and a fall back to another device
 *     (runtime/Executor.cpp:15,56-59; runtime/Scheduler.cpp:221-252).
 *   - Arrays are row-major: W is the number of columns, H the number of rows
 *     (api/ArrayFun.cpp:74-90).  Vectorised traces stack `slots` arrays of
 *     W x H elements back to back.
 *   - Device buffers are owned by the context and named by a 64-bit id the
 *     host chooses (the reference keys them by trace hash and variable,
 *     memmgr/MemTrans.hpp:48-51).  Host memory stays the caller's.
 *   - chai_cuda_evaluate is called from one thread per context (one CUDA
 *     stream per context); readback / release may come from any thread
 *     (memmgr/MemTrans.hpp:43-47 guards the same way with _memMutex).
 *   - There is no CPU fallback inside this library: without a usable B200
 *     every entry point that would compute returns CHAI_ERR_NO_DEVICE.
 */
#ifndef CHAI_B200_H
#define CHAI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAI_B200_ABI_VERSION 2

typedef enum chai_status {
    CHAI_OK = 0,
    CHAI_ERR_INVALID = -1,      /* bad argument or malformed trace */
    CHAI_ERR_UNSUPPORTED = -2,  /* opcode / shape / precision not handled */
    CHAI_ERR_OOM = -3,          /* device allocation failed */
    CHAI_ERR_LAUNCH = -4,       /* kernel launch or execution failed */
    CHAI_ERR_TIMEOUT = -5,      /* a bounded device wait gave up (status word set) */
    CHAI_ERR_NOT_FOUND = -6,    /* unknown buffer id */
    CHAI_ERR_NO_DEVICE = -7,    /* no CUDA device / not an sm_100 part */
    CHAI_ERR_JIT = -8,          /* runtime compilation of a trace kernel failed */
    CHAI_ERR_INJECTED = -9      /* failure forced by CHAI_FAULT_INJECT (testing) */
} chai_status;

/* Precision codes, as misc/PrecType.hpp numbers them. */
enum { CHAI_U32 = 0, CHAI_I32 = 1, CHAI_F32 = 4, CHAI_F64 = 8 };

/* RNG variants, as api/chai.h:412-417 numbers them. */
enum { CHAI_RNG_PHILOX = 1230, CHAI_RNG_THREEFRY = 1231 };

typedef struct chai_cuda_ctx chai_cuda_ctx;

/* ------------------------------------------------------------------ life */

/* Replaces Translator::initDevice / DeviceBase::initDevice
 * (runtime/DeviceBase.hpp:22-61, runtime/Translator.cpp:353-364).
 * `config` is the text of a device spec (devspec.cfg keywords are accepted and
 * ignored where meaningless on CUDA); recognised keys, one per line or
 * space-separated, `Key=Value`:
 *   GemmPrecision=auto|fp32|tf32|bf16|bf16x3|bf16x6|fp8   f32 matmul arithmetic
 *                         (auto, the default: bf16x3 on the tensor cores for
 *                         M, N >= 32 and K >= 16, FP32 CUDA cores otherwise)
 *   RngPi=<double>        constant inside Box-Muller (default 3.14159, the
 *                         value the reference JIT prints)
 *   RngLayout=chai|counter   key/counter placement (default chai)
 *   TunerMode=learned|exhaustive|off, TuneDB=<path>
 *   JitCache=<dir>        on-disk cache of compiled trace kernels
 * May be NULL. */
int chai_cuda_init(int device, const char* config, chai_cuda_ctx** out);
/* Clean shutdown: frees every buffer, module and stream (no ShutdownNOP). */
int chai_cuda_shutdown(chai_cuda_ctx* ctx);
int chai_cuda_synchronize(chai_cuda_ctx* ctx);
const char* chai_cuda_error_string(int status);
/* Failure-detection self-test: one kernel waits on a shared-memory mbarrier
 * that nothing arrives on, with the bounded wait every persistent kernel of
 * this library uses (try_wait in a loop limited by %globaltimer); after
 * `limit_ms` (0 < limit_ms <= 2000) it gives up and writes the context status
 * word, so the call returns CHAI_ERR_TIMEOUT and the context stays usable.
 * No counterpart in the reference (its device code has no waits). */
int chai_cuda_selftest_wait(chai_cuda_ctx* ctx, double limit_ms);

/* Human-readable detail of the last failure on this context. */
const char* chai_cuda_last_error(chai_cuda_ctx* ctx);
/* Device time of a hot kernel ("gemm_tc", "trace", "gemv") accumulated over
 * its launches, measured with CUDA events on the context stream when the
 * process runs with CHAI_KERNEL_TIMING=1 (the counterpart of the reference's
 * per-dispatch timing, runtime/Scheduler.cpp:198-220).  The name
 * "plan_replay" reports in *launches the number of evaluations replayed from
 * the plan cache (config PlanCache=1, the default: a trace whose cells,
 * scalars, shapes and bindings repeat an earlier one re-issues its recorded
 * device operations on its own buffers without translating again);
 * "grouped_fused" the number of grouped GEMMs whose f32 operands were split
 * inside the GEMM kernel (config GroupedSplit=fused, the default). */
int chai_cuda_kernel_stats(chai_cuda_ctx* ctx, const char* name, double* total_ms, uint64_t* launches,
                           int reset);
/* Run subsequent work on an external cudaStream_t (NULL = the context's own). */
int chai_cuda_set_stream(chai_cuda_ctx* ctx, void* cuda_stream);

/* ---------------------------------------------------------------- memory */

/* Replace MemTrans::memalloc / MemCallback::swizzle / untrackMem
 * (memmgr/MemTrans.hpp:31-235, common/MemCallback.hpp:13-21). */
int chai_cuda_buffer_alloc(chai_cuda_ctx* ctx, uint64_t id, size_t bytes);
/* Register caller-owned device memory under `id` (never freed by the library). */
int chai_cuda_buffer_wrap(chai_cuda_ctx* ctx, uint64_t id, void* device_ptr, size_t bytes);
int chai_cuda_buffer_info(chai_cuda_ctx* ctx, uint64_t id, void** device_ptr, size_t* bytes);
/* Host -> device copy of `bytes` at offset 0; the host buffer may be pageable. */
int chai_cuda_upload(chai_cuda_ctx* ctx, uint64_t id, const void* host, size_t bytes);
/* Device -> host copy; waits for all work on the context that writes `id`. */
int chai_cuda_readback(chai_cuda_ctx* ctx, uint64_t id, void* host, size_t bytes);
int chai_cuda_release(chai_cuda_ctx* ctx, uint64_t id);
/* Device -> device copy of `bytes` from buffer `src` into buffer `dst`
 * (allocated when missing), ordered on the context stream: the copy the
 * reference's memory manager makes when a value must survive an in-place
 * update (memmgr/MemTrans.hpp:31-235). */
int chai_cuda_buffer_copy(chai_cuda_ctx* ctx, uint64_t dst, uint64_t src, size_t bytes);

/* ----------------------------------------------------------------- trace */

/* One bytecode cell, mirroring chai_internal::BC (bytecode/BC.hpp:15-36). */
enum { CHAI_BC_OPCODE = 0, CHAI_BC_VARIABLE = 1, CHAI_BC_SCALAR = 2, CHAI_BC_MEMORY = 3, CHAI_BC_KERNEL = 4 };
typedef struct chai_bc {
    uint32_t kind;      /* CHAI_BC_* */
    uint32_t code;      /* opcode (ByteCodes.hpp numbers) or variable number */
    uint32_t version;   /* variable version */
    uint32_t reserved;
    double   scalar;    /* CHAI_BC_SCALAR payload */
    uint64_t buffer;    /* CHAI_BC_MEMORY: buffer id standing for a FrontMem box */
} chai_bc;

/* One statement: the bytecode stack of an assignment, in push order (operands
 * are pushed last-argument first, the opcode last: api/ArrayFun.cpp:44-52). */
typedef struct chai_stmt {
    uint32_t lhs_variable;
    uint32_t lhs_version;
    uint32_t n_cells;
    uint32_t reserved;
    const chai_bc* cells;
} chai_stmt;

/* A vectorised trace (common/VectorTrace.hpp:28-119). */
/* Inline OpenCL kernel of a trace: ProgramCL (api/ProgramCL.cpp; the
 * reference records it as the statement [AstOpenCL box, kernel_from_opencl]
 * and prints / enqueues it in jitast/AstOpenCL.cpp, enqueue/EnqueueOpenCL.cpp).
 * Here the statement is [{CHAI_BC_KERNEL, .buffer = index into
 * chai_trace_desc.kernels}, opcode 50]; the OpenCL C text is compiled for
 * sm_100a by NVRTC through a prelude that maps the OpenCL work-item functions,
 * address-space qualifiers and barrier onto CUDA.  Array arguments are the
 * arrays' device storage, updated in place: statements after the kernel read
 * the updated values under the same (variable, version), as in the
 * reference.  Scalar OpenCL C only (no vector types, no image2d_t). */
enum { CHAI_KARG_ARRAY = 0, CHAI_KARG_LOCAL = 1, CHAI_KARG_SCALAR = 2 };
typedef struct chai_kernel_arg {
    uint32_t kind;              /* CHAI_KARG_* */
    uint32_t prec;              /* element / scalar precision: CHAI_U32, CHAI_I32, CHAI_F32, CHAI_F64 */
    uint32_t variable;          /* ARRAY: the array variable and its current version */
    uint32_t version;
    double   value;             /* SCALAR: the value; LOCAL: number of elements */
} chai_kernel_arg;
typedef struct chai_inline_kernel {
    const char* source;         /* the whole OpenCL C program text */
    const char* name;           /* the __kernel function to run */
    uint32_t n_args;
    uint32_t reserved;
    const chai_kernel_arg* args;
    uint64_t global_size[2];    /* work items per dimension; global_size[1] = 0 for 1-D */
    uint64_t local_size[2];     /* work-group size per dimension (divides global_size) */
} chai_inline_kernel;

typedef struct chai_trace_desc {
    uint32_t num_traces;        /* slots: identical traces batched together */
    uint32_t n_stmts;
    const chai_stmt* stmts;
    uint64_t hash;              /* front-end trace hash (0: computed here) */
    const chai_inline_kernel* kernels;   /* inline kernels the statements refer to (may be NULL) */
    uint32_t n_kernels;
    uint32_t reserved;
} chai_trace_desc;

/* Variables that live outside the trace: inputs computed by earlier traces and
 * outputs later traces or the host read (the reference's liveVariables and
 * BackMem boxes, common/VectorTrace.hpp:33-76). */
typedef struct chai_buffer_binding {
    uint32_t variable;
    uint32_t prec;              /* CHAI_U32 .. CHAI_F64 */
    uint64_t width, height;
    uint32_t slots;
    uint32_t reserved;
    uint64_t buffer;            /* buffer id holding slots*height*width elements */
} chai_buffer_binding;

/* Replaces Translator::sub_evaluate (runtime/Translator.cpp:366-411). */
int chai_cuda_evaluate(chai_cuda_ctx* ctx, const chai_trace_desc* trace,
                       const chai_buffer_binding* bindings, size_t n_bindings);

/* Diagnostic counterpart of the reference's logged kernel source
 * (kernel/KernelCache.cpp:82-89 prints generated OpenCL under --log): plans
 * the trace, emits every fused element kernel as CUDA C and compiles each with
 * NVRTC for sm_100a.  Needs no device; allocates and launches nothing.  The
 * generated source (or the error text on failure) is copied to `out`
 * (NUL-terminated, truncated to `cap`); `needed` receives its full size. */
int chai_cuda_trace_source(const chai_trace_desc* trace, const chai_buffer_binding* bindings,
                           size_t n_bindings, const char* config, char* out, size_t cap, size_t* needed);

/* The value each assignment statement of a trace produces: its left-hand side
 * and the precision, shape and slots of the right-hand side, in statement order
 * (read-back statements and inline kernels produce none).  Input shapes come
 * from `bindings`.  Parses only: needs no device, allocates and launches
 * nothing.  A device adapter uses it to size the host memory of the variables
 * a trace leaves live, as the reference's memory manager sizes the BackMem of
 * a live variable (memmgr/MemTransPrivate.cpp:45-140).  `*count` receives the
 * number of values; at most `cap` are written. */
typedef struct chai_value_shape {
    uint32_t variable, version;     /* the statement's left-hand side */
    uint32_t prec, slots;
    uint64_t width, height;
} chai_value_shape;
int chai_cuda_trace_shapes(const chai_trace_desc* trace, const chai_buffer_binding* bindings, size_t n_bindings,
                           chai_value_shape* out, size_t cap, size_t* count);

/* Many traces of uneven length in one persistent launch captured in a CUDA
 * graph.  All traces share one bytecode program (same hash, different W/H);
 * trace i reads/writes buffers bindings[i*n_per .. ]; scalar results land in
 * results[i] (host memory).  Replaces the per-hash VectorTrace batching of
 * runtime/Scheduler.cpp:48-89, which only batches equal shapes. */
int chai_cuda_evaluate_many(chai_cuda_ctx* ctx, const chai_trace_desc* const* traces, size_t n_traces,
                            double* results);

/* --------------------------------------------------------- direct kernels */

/* Chai random array fill (Random123/R123Philox.cpp:288-523 and
 * R123Threefry.cpp:289-535 as called from kernel/Function.cpp:433-503). */
typedef struct chai_rng_desc {
    uint32_t variant;           /* CHAI_RNG_PHILOX / CHAI_RNG_THREEFRY */
    uint32_t prec;              /* CHAI_U32, CHAI_I32, CHAI_F32, CHAI_F64 */
    uint32_t dist;              /* 0 uniform, 1 normal */
    uint32_t vec_len;           /* 4 (32-bit default), 2 (f64 default) or 1 */
    uint64_t seed;              /* generator seed at the call (counter word 0) */
    uint64_t width, height;
    uint32_t slots;
    uint32_t has_limits;        /* uniform f32/f64: u*(max-min)+min */
    double   min_limit, max_limit;
} chai_rng_desc;
int chai_cuda_rng_fill(chai_cuda_ctx* ctx, const chai_rng_desc* d, void* device_out);

/* GEMM C = alpha * op(A) op(B) + beta * C  (EnqueueMatmulAuto.cpp:21-404,
 * autotune/EvergreenMatmulMM.cpp).  Row-major, lda/ldb/ldc in elements. */
enum {
    CHAI_GEMM_FP32 = 0,     /* CUDA-core FFMA, f32 accumulate */
    CHAI_GEMM_TF32 = 1,     /* tcgen05 kind::tf32 */
    CHAI_GEMM_BF16 = 2,     /* operands rounded to bf16, tcgen05 kind::f16 */
    CHAI_GEMM_BF16X3 = 3,   /* fp32 split hi+lo bf16, 3 products */
    CHAI_GEMM_BF16X6 = 4,   /* fp32 split hi+mid+lo bf16, 6 products */
    CHAI_GEMM_FP8 = 5,      /* e4m3 with per-128x128-tile scales */
    CHAI_GEMM_FP64 = 6,     /* f64 operands (Arrayd64), CUDA-core DFMA */
    CHAI_GEMM_AUTO = 7      /* context default (GemmPrecision; auto: by shape) */
};
typedef struct chai_gemm_desc {
    int32_t  precision;         /* CHAI_GEMM_* */
    int32_t  trans_a, trans_b;
    int32_t  reserved;
    int64_t  m, n, k;
    const void* a; int64_t lda;
    const void* b; int64_t ldb;
    void*    c;    int64_t ldc;
    double   alpha, beta;
    int64_t  batch;             /* >= 1: strided batch (traces / slots) */
    int64_t  stride_a, stride_b, stride_c;
} chai_gemm_desc;
int chai_cuda_gemm(chai_cuda_ctx* ctx, const chai_gemm_desc* d);

/* The same GEMM with a, b and c in HOST memory (pinned memory copies fastest):
 * the host-resident matmul operands and read-back of the reference's memory
 * manager (memmgr/MemTransJIT.cpp:18-327) overlapped with the GEMM.  B is
 * uploaded once; A goes up in blocks of `block_rows` rows (0: about an eighth
 * of M, whole 128-row tiles) on a copy stream, each block's GEMM runs on the
 * context stream as its rows land, and its rows of C come back on a second
 * copy stream during the next block.  C is bit-identical to uploading the
 * operands and calling chai_cuda_gemm.  One problem (batch <= 1), no
 * transposes; returns when C is in host memory. */
int chai_cuda_gemm_host(chai_cuda_ctx* ctx, const chai_gemm_desc* d, int64_t block_rows);

/* y = alpha * op(A) x + beta * y, f32 or f64 (autotune/EvergreenMatmulMV.cpp). */
int chai_cuda_gemv(chai_cuda_ctx* ctx, uint32_t prec, int trans, int64_t m, int64_t n, double alpha,
                   const void* a, int64_t lda, const void* x, double beta, void* y);

/* Many independent f32 GEMMs of different shapes in one persistent
 * tensor-core launch (C_i = A_i B_i, row-major, packed; the reference runs
 * one matmul statement per trace, enqueue/EnqueueMatmulAuto.cpp:21-404).
 * precision: bf16, bf16x3 or bf16x6 (fp32 and AUTO-with-fp32 mean bf16x3).
 * When every A and B is 16-byte aligned and every K and N is a multiple of 4,
 * the kernel splits the f32 operands into bf16 planes itself; otherwise the
 * planes go through HBM first.  Both paths give bit-identical C.  The tile
 * records are rebuilt only when the problem array changes. */
typedef struct chai_gemm_problem {
    int32_t m, n, k, reserved;
    const float* a; const float* b; float* c;
} chai_gemm_problem;
int chai_cuda_gemm_grouped(chai_cuda_ctx* ctx, int32_t precision, const chai_gemm_problem* problems,
                           int32_t count);

/* sum / mean / dot_product over `slots` arrays of n elements each
 * (enqueue/EnqueueReduce.cpp:21-222; interp/InterpAccum.cpp:13-70).
 * op: 0 sum, 1 mean, 2 dot_product (b used).  Results (one per slot) are
 * written as doubles to host memory `out`; at most 4096 slots per call. */
int chai_cuda_reduce(chai_cuda_ctx* ctx, uint32_t op, uint32_t prec, const void* a, const void* b,
                     uint64_t n, uint32_t slots, double* out);

/* Allocation-free variant of chai_cuda_reduce.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory at
 * call time (a fixed arena owns the GPU, or an allocation could block or fail
 * late).  It needs no context and calls no allocator; the caller passes the
 * inputs and a device output of `slots` doubles, and the kernels run on
 * `cuda_stream` (NULL: the legacy default stream).  Partial sums live in a
 * fixed device array of 8192 doubles that every GPU loading the library keeps
 * until exit, so at most 8192 slots are accepted (CHAI_ERR_UNSUPPORTED
 * beyond).  All calls share that array: calls whose kernels overlap on the GPU
 * race.  The kernels run in the calling thread's current CUDA context (the
 * device's primary context unless the caller made its own driver-API context
 * current); the first call in a context looks up the array's address there,
 * so make that first call before any stream capture.  n = 0 gives 0 for sum
 * and dot_product and NaN (0/0) for mean.  CHAI_ERR_LAUNCH reports a failure
 * of this call's own launches only. */
int chai_cuda_reduce_noalloc(uint32_t op, uint32_t prec, const void* a, const void* b, uint64_t n,
                             uint32_t slots, double* device_out, void* cuda_stream);

/* ------------------------------------------------------------------ tuner */

/* Replace StandardEM / AutoTuneEM / AutoTuneBench (autotune/StandardEM.cpp:69-147,
 * autotune/AutoTuneBench.cpp:17-251) and the journal (autotune/AutoTuneMemo.hpp). */
typedef struct chai_gemm_key {
    int64_t m, n, k;
    int32_t precision;          /* CHAI_GEMM_* */
    int32_t is_gemv;
} chai_gemm_key;
/* GEMM: block_m 128 (one CTA per tile, block_n 64|128|256) or 256 (a CTA pair
 * on two SMs, tcgen05 cta_group::2, cluster 2 x 1, block_n 128|256), block_k
 * 128 bytes, stages (shared-memory pipeline depth), group_m (tile-raster strip
 * height).  GEMV: block_m = warps (rows) per block, vec_width = 16-byte loads
 * in flight per lane; block_m = 0 is the bulk-copy kernel (A streamed through
 * shared memory, 16-byte aligned operands). */
typedef struct chai_gemm_cfg {
    int32_t block_m, block_n, block_k, stages;
    int32_t vec_width, cluster_m, cluster_n, group_m;
    double  measured_us;        /* timing of the configuration (0 if not timed) */
} chai_gemm_cfg;
enum { CHAI_TUNE_LEARNED = 0, CHAI_TUNE_EXHAUSTIVE = 1, CHAI_TUNE_DEFAULT = 2 };
/* Choose a configuration for `key` and remember it (used by later GEMM/GEMV
 * calls of that shape).  EXHAUSTIVE times every configuration of the search
 * space (AutoTuneBench); LEARNED ranks them with the MLP cost model and times
 * only the top k (TopK in the init config, default 3).  DEFAULT returns,
 * untimed and unremembered, the configuration an untuned call of that shape
 * uses (the method without the tuner). */
int chai_cuda_tune(chai_cuda_ctx* ctx, const chai_gemm_key* key, int mode, chai_gemm_cfg* out);
/* Time every configuration of the search space for `key` (the exhaustive
 * sweep that generates the cost model's training data). */
int chai_cuda_tune_sweep(chai_cuda_ctx* ctx, const chai_gemm_key* key, chai_gemm_cfg* out, int cap, int* n);
/* The 14 cost-model input features of (key, cfg) into out[0..13]. */
#define CHAI_TUNE_FEATURES 14
int chai_cuda_tune_features(const chai_gemm_key* key, const chai_gemm_cfg* cfg, float* out);
/* Tuning DB / journal: best configuration per key, plus the MLP weights. */
int chai_cuda_tune_db_load(chai_cuda_ctx* ctx, const char* path);
int chai_cuda_tune_db_save(chai_cuda_ctx* ctx, const char* path);

/* MLP cost model (14 features -> 128 -> 128 -> 128 -> 1, ReLU), trained on the
 * GPU by this library's forward / backward / Adam kernels on measured
 * (key, cfg, measured_us) samples; the target is log(measured_us). */
int chai_cuda_mlp_train(chai_cuda_ctx* ctx, const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n,
                        int epochs, double lr, uint64_t seed, double* final_loss);
int chai_cuda_mlp_predict(chai_cuda_ctx* ctx, const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n,
                          double* log_us);
/* Loss and gradient of every weight for the current weights (no update). */
int chai_cuda_mlp_gradients(chai_cuda_ctx* ctx, const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n,
                            float* grads, size_t cap, double* loss);
/* Get (set = 0) or set (set = 1) all weights, in the order W1 b1 W2 b2 W3 b3
 * W4 b4 (W row-major in x out), plus the target's mean and scale last;
 * *count receives the number of floats. */
int chai_cuda_mlp_weights(chai_cuda_ctx* ctx, float* buf, size_t cap, size_t* count, int set);

#ifdef __cplusplus
}
#endif

#endif
