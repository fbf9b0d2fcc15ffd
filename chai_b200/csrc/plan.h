// Recorded launch plans of traces (the plan cache).
//
// The reference compiles a trace once per hash and keeps the kernels
// (kernel/KernelCache.cpp:23-42, enqueue/JustInTimeMemo.hpp:28-130) but
// re-runs its whole bytecode -> AST -> statement pipeline on every evaluation
// (runtime/Translator.cpp:366-411).  Here the first evaluation of a trace
// records every device operation it issues with the provenance of each
// device pointer; a later evaluation of a trace with the same structure
// (cells, scalars, shapes, bindings; buffer ids may differ) replays the
// operations with the pointers of its own buffers, skipping parsing,
// planning, code generation and compilation.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "chai_b200.h"

namespace chai {

// Where a device pointer comes from.
struct Ref {
    enum Kind : uint8_t { NONE, BUFFER, TEMP, SCRATCH, STATUS } kind = NONE;
    uint32_t idx = 0;      // BUFFER: ordinal in the trace's buffer list; TEMP: temporary index
    uint64_t off = 0;      // byte offset inside it
    void* raw = nullptr;   // the pointer itself (used by the recording run)
};

struct TmapRec {
    bool encode = false;   // false: an all-zero map (kernel uses wrapped loads only)
    CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    uint64_t dims[3] = {0, 0, 0}, strides[2] = {0, 0};
    uint32_t box[3] = {0, 0, 0};
    Ref base;
};

struct Step {
    enum Kind { KERNEL, COMBINE, GEMM, GEMV, TRANSPOSE, COPY, COPY2D, MEMSET } kind = KERNEL;
    // KERNEL (runtime-compiled trace kernel)
    void* fn = nullptr;
    dim3 grid, block;
    struct Arg {
        enum Kind : uint8_t { I64, PTR, TMAP } kind = I64;
        long long v = 0;
        Ref r;
        int map = -1;
    };
    std::vector<Arg> args;
    std::vector<TmapRec> maps;
    size_t smem = 0;                // dynamic shared memory bytes
    size_t scratch_need = 0;        // ensure_scratch before the step
    // COMBINE
    int nblocks = 0, nred = 0, slots = 0;
    Ref partials;
    std::vector<Ref> outs;
    std::vector<int> precs;
    std::vector<double> scales;
    // GEMM
    chai_gemm_desc desc{};
    // GEMM / GEMV / TRANSPOSE / COPY / COPY2D / MEMSET operands
    Ref a, b, c;
    uint32_t prec = 0;
    int trans = 0;
    int64_t m = 0, n = 0, lda = 0, w = 0, h = 0, nslots = 0;
    double alpha = 1, beta = 0;
    size_t bytes = 0, dpitch = 0, spitch = 0, width = 0, height = 0;
    int value = 0;
};

struct Plan {
    std::vector<uint64_t> key;      // full key material (compared on lookup)
    std::vector<Step> steps;
    std::vector<size_t> temp_bytes; // temporaries, allocated in this order on replay
    std::vector<size_t> buf_alloc;  // per buffer ordinal: bytes the evaluation allocates (0: none)
    std::vector<size_t> buf_need;   // per buffer ordinal: bytes the evaluation reads as input (0: none)
    size_t kernels = 0;
};

// Key material of a trace + bindings, and its buffer ids in canonical order
// (bindings in the given order, then MEMORY cells in statement / cell order,
// first occurrence of each id).
void plan_key(const chai_trace_desc* t, const chai_buffer_binding* b, size_t nb, std::vector<uint64_t>& key,
              std::vector<uint64_t>& ids);

}  // namespace chai
