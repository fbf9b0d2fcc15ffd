// Trace translator internals (see trace.cpp).
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "chai_b200.h"
#include "plan.h"

struct chai_cuda_ctx;

namespace chai {

struct Node {
    // INLINE: an inline OpenCL kernel (buffer = its index in the trace's kernel
    // table, kids = its array arguments); AFTER: an array argument's value once
    // the kernel has run (kids = {INLINE, value before}; same storage)
    enum Kind { VAR, INPUT, SCALAR, OP, CONVERT, RNG, INDEX, FILL, MAKE, READ, MATMUL, MATMULG, TRANSPOSE,
                REDUCE, GATHER, INLINE, AFTER } kind = OP;
    uint32_t op = 0;
    int prec = CHAI_F32;
    uint64_t W = 1, H = 1;
    uint32_t slots = 1;
    std::vector<int> kids;
    double scalar = 0;
    uint32_t var = 0, ver = 0;
    uint64_t buffer = 0;            // MAKE / READ / INPUT buffer id
    int read_kind = 0;              // 0 read_scalar, 1 read1, 2 read2
    // RNG
    uint32_t variant = CHAI_RNG_PHILOX, dist = 0;
    uint64_t seed = 0;
    bool limits = false;
    double lo = 0, hi = 1;
    // INDEX
    int dim = 0;
    // MATMULG
    double alpha = 1, beta = 0;
    // storage when materialised
    void* dev = nullptr;
    uint64_t storage_buffer = 0;
};

class Translator {
public:
    // dry: plan and compile every kernel, allocate and launch nothing
    explicit Translator(chai_cuda_ctx* ctx, bool dry = false) : ctx_(ctx), dry_(dry) {}
    ~Translator();
    int run(const chai_trace_desc* t, const chai_buffer_binding* b, size_t nb);
    // steps 1-2 of run(): parse the statements with the bindings' input shapes
    int parse_all(const chai_trace_desc* t, const chai_buffer_binding* b, size_t nb);
    // after parse_all(): the value each assignment statement produces, in order
    const std::vector<chai_value_shape>& statement_values() const { return stmt_values_; }
    // parse the statements only (no bindings, storage or launches)
    int parse_only(const chai_trace_desc* t);
    // root node of the last assignment when it is a reduction, else -1
    int result_root() const;
    // after run(): value of result_root() as a double (host)
    int read_result(double* out);
    // scalar results of reductions that are statement roots (for evaluate_many)
    const std::vector<Node>& nodes() const { return nodes_; }
    // generated source of the last element kernel (diagnostics / tests)
    std::string last_source;
    std::string all_sources;
    size_t kernels_launched = 0;

    // plan cache (plan.h): record the device operations of this run with the
    // provenance of their pointers, or replay a recorded plan
    void begin_record(const std::vector<uint64_t>& buffer_ids);
    std::unique_ptr<Plan> take_plan();          // null when the run is not replayable
    // 0: replayed; > 0: the plan does not fit these buffers (translate instead); < 0: error
    int replay(const Plan& p, const std::vector<uint64_t>& buffer_ids);

private:
    chai_cuda_ctx* ctx_;
    bool dry_ = false;
    std::vector<Node> nodes_;
    std::map<uint32_t, chai_buffer_binding> bindings_;
    std::map<std::pair<uint32_t, uint32_t>, int> assigned_;
    std::map<uint32_t, int> latest_;
    std::map<uint32_t, int> inputs_;
    std::map<std::string, int> cse_;
    std::vector<std::pair<uint32_t, int>> stmt_roots_;
    std::vector<chai_value_shape> stmt_values_;
    int first_inline_ = -1;
    std::vector<int> reads_;
    std::vector<bool> materialize_;
    std::vector<void*> temps_;
    uint32_t slots_ = 1;
    uint32_t unsupported_op_ = 0;
    // plan recording / replay
    bool recording_ = false, replaying_ = false, cacheable_ = true;
    std::unique_ptr<Plan> plan_;
    std::vector<uint64_t> buf_ids_;
    std::vector<size_t> temp_sizes_;
    Ref ref_of(const void* p);
    void* ptr_of(const Ref& r) const;
    void note_buffer(uint64_t id, size_t bytes, bool alloc);
    int exec(Step& s);
    int run_step(const Step& s);

    int fail(int st, const std::string& msg);
    int add(Node n);
    double scalar_cell(const chai_stmt& s, int& pos, bool& ok);
    int parse(const chai_stmt& s, int& pos);
    int resolve_var(const Node& v);
    size_t node_bytes(const Node& n) const;
    int assign_storage(int i);
    int schedule(const std::vector<int>& order);
    int emit_group(const std::vector<int>& roots);
    int emit_linalg(int i);
    int do_read(int i);
    int emit_inline(int i);
    const chai_inline_kernel* kernels_ = nullptr;
    uint32_t n_kernels_ = 0;
};

// OpenCL C program text -> CUDA source (inline_cl.cpp)
int opencl_to_cuda(const std::string& src, const std::string& name, const std::vector<size_t>& local_counts,
                   int work_dim, std::string& out, std::string& err, std::vector<char>* image_args = nullptr,
                   size_t* local_bytes = nullptr);

}  // namespace chai
