// Trace translator: chai bytecode -> fused sm_100a kernels.
//
// The B200 counterpart of Translator::sub_evaluate (runtime/Translator.cpp:
// 366-411).  The reference pipeline is ByteTrace (constant lifting, loop
// rolling) -> AST -> statement list -> WorkTrace::reorder/together (group
// statements into "ID spaces", elide internal variables, keep temporaries in
// registers) -> OpenCL printers -> clBuildProgram -> enqueue.  Here:
//
//   1. parse   every statement's bytecode stack into a node DAG
//              (api/*Fun.cpp push orders), resolving variable references to
//              the producing statement or to a bound input buffer;
//   2. infer   shape (W, H, slots) and precision (widest operand wins,
//              interp/InterpFun2.cpp:21) bottom-up (api/ArrayFun.cpp:54-119);
//   3. choose  what lives in HBM: bound outputs, read-backs, matmul/transpose
//              operands and results, gather sources and reductions -- every
//              other value stays in registers (ElideInternal/UseRegister);
//   4. group   materialisation roots with the same iteration space into one
//              kernel unless one needs another complete first (a gather
//              source or a reduction result) -- the "together" pass;
//   5. emit    each element group as CUDA C built on chai_trace_prelude.cuh,
//              compile it with NVRTC (cached by source hash) and launch it;
//              matmul, GEMV and transpose go to the static kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <set>
#include <sstream>

#include "internal.h"
#include "jit.h"
#include "trace.h"

namespace chai {

// ------------------------------------------------------------ op tables
static int arity_of(uint32_t op)
{
    switch (op) {
        case 1: case 2: case 3: case 4: case 10: case 15: case 16: case 122: case 131: case 132:
        case 200: case 201: case 202: case 203: case 204: case 205: case 206: case 208: case 209:
        case 211: case 212: case 214: case 215: case 216: case 217: case 218: case 219: case 220:
        case 221: case 222: case 223: case 225: case 233: case 235: case 237: case 238: case 239:
        case 240: case 241: case 246: case 253: case 255: case 256: case 257: case 259: case 260:
        case 261: case 262: case 263: case 264: case 265: case 266: case 301: case 305: case 308:
        case 400: case 404: case 507: case 508: case 509: case 510: case 513:
            return 1;
        case 11: case 12: case 13: case 14: case 17: case 18: case 19: case 20: case 21: case 22:
        case 30: case 31: case 32: case 33: case 34: case 35: case 36: case 37: case 40: case 120:
        case 130: case 207: case 210: case 213: case 224: case 227: case 228: case 229: case 232:
        case 234: case 243: case 244: case 247: case 248: case 249: case 250: case 251: case 254:
        case 302: case 303: case 306: case 401: case 402: case 405: case 411: case 412: case 413:
        case 414: case 415: case 500: case 501: case 502: case 503: case 504: case 505: case 506:
        case 511: case 512:
            return 2;
        case 23: case 41: case 226: case 242: case 300: case 304: case 307: case 406: case 407: case 408:
            return 3;
    }
    return -1;
}

static bool is_int_only(uint32_t op)
{
    switch (op) {
        case 15: case 18: case 19: case 20: case 21: case 22: case 404: case 401: case 402: case 405:
        case 411: case 412: case 413: case 414: case 415: case 406: case 407: case 408:
            return true;
    }
    return false;
}

static bool fp_only(uint32_t op)
{
    return (op >= 200 && op <= 299) || op == 301 || op == 304 || op == 305 || op == 306 || op == 307 ||
           op == 308 || (op >= 506 && op <= 513);
}

static const char* ctype(int prec)
{
    switch (prec) {
        case CHAI_U32: return "unsigned";
        case CHAI_I32: return "int";
        case CHAI_F32: return "float";
        case CHAI_F64: return "double";
    }
    return "float";
}

static int wider(int a, int b) { return a > b ? a : b; }

// ---------------------------------------------------------------- parse
int Translator::fail(int st, const std::string& msg) { return set_error(ctx_, st, msg); }

// Hash-consing: a subexpression pushed more than once (an ArrayExp object
// used in several places pushes its whole bytecode each time) becomes one
// node, computed once per element in the fused kernel.  Random arrays are
// included: identical RNG cells name the same array (each rng_*_make call
// advances the generator's seed, api/RngFun.cpp:30), so sharing is exact.
int Translator::add(Node n)
{
    if (n.kind != Node::READ) {
        std::ostringstream k;
        uint64_t sb, lb, hb, ab, bb;
        memcpy(&sb, &n.scalar, 8); memcpy(&lb, &n.lo, 8); memcpy(&hb, &n.hi, 8);
        memcpy(&ab, &n.alpha, 8); memcpy(&bb, &n.beta, 8);
        k << (int)n.kind << ':' << n.op << ':' << n.prec << ':' << n.W << ':' << n.H << ':' << n.slots << ':' << sb
          << ':' << n.var << ':' << n.ver << ':' << n.buffer << ':' << n.variant << ':' << n.dist << ':' << n.seed
          << ':' << n.limits << ':' << lb << ':' << hb << ':' << n.dim << ':' << ab << ':' << bb << '|';
        for (int kid : n.kids) k << kid << ',';
        auto it = cse_.find(k.str());
        if (it != cse_.end()) return it->second;
        nodes_.push_back(n);
        cse_[k.str()] = (int)nodes_.size() - 1;
        return (int)nodes_.size() - 1;
    }
    nodes_.push_back(n);
    return (int)nodes_.size() - 1;
}

double Translator::scalar_cell(const chai_stmt& s, int& pos, bool& ok)
{
    if (pos < 0 || s.cells[pos].kind != CHAI_BC_SCALAR) {
        ok = false;
        return 0;
    }
    return s.cells[pos--].scalar;
}

int Translator::parse(const chai_stmt& s, int& pos)
{
    if (pos < 0) return -1;
    const chai_bc& c = s.cells[pos--];
    if (c.kind == CHAI_BC_VARIABLE) {
        Node n;
        n.kind = Node::VAR;
        n.var = c.code;
        n.ver = c.version;
        return resolve_var(n);
    }
    if (c.kind != CHAI_BC_OPCODE) return -1;
    const uint32_t op = c.code;
    bool ok = true;
    Node n;
    n.op = op;
    if (op >= 1 && op <= 4) {
        n.kind = Node::CONVERT;
        int k = parse(s, pos);
        if (k < 0) return -1;
        n.kids = {k};
        n.prec = op == 1 ? CHAI_U32 : op == 2 ? CHAI_I32 : op == 3 ? CHAI_F32 : CHAI_F64;
        if (nodes_[k].prec == n.prec) return k;   // identity conversion (every assignment ends in one)
        n.W = nodes_[k].W; n.H = nodes_[k].H; n.slots = nodes_[k].slots;
        return add(n);
    }
    if (op >= 5 && op <= 8) {
        n.kind = Node::SCALAR;
        n.scalar = scalar_cell(s, pos, ok);
        n.prec = op == 5 ? CHAI_U32 : op == 6 ? CHAI_I32 : op == 7 ? CHAI_F32 : CHAI_F64;
        return ok ? add(n) : -1;
    }
    if ((op >= 42 && op <= 49)) {
        n.kind = Node::INDEX;
        const bool two = op >= 46;
        n.dim = (int)scalar_cell(s, pos, ok);
        n.W = (uint64_t)scalar_cell(s, pos, ok);
        n.H = two ? (uint64_t)scalar_cell(s, pos, ok) : 1;
        const int k = (op - 42) % 4;
        n.prec = k == 0 ? CHAI_U32 : k == 1 ? CHAI_I32 : k == 2 ? CHAI_F32 : CHAI_F64;
        return ok ? add(n) : -1;
    }
    if (op >= 60 && op <= 67) {
        n.kind = Node::MAKE;
        n.W = (uint64_t)scalar_cell(s, pos, ok);
        n.H = (uint64_t)scalar_cell(s, pos, ok);
        n.slots = (uint32_t)scalar_cell(s, pos, ok);
        if (!ok || pos < 0 || s.cells[pos].kind != CHAI_BC_MEMORY) return -1;
        n.buffer = s.cells[pos--].buffer;
        const int k = (op - 60) % 4;
        n.prec = k == 0 ? CHAI_U32 : k == 1 ? CHAI_I32 : k == 2 ? CHAI_F32 : CHAI_F64;
        return add(n);
    }
    if (op >= 68 && op <= 82) {
        // ones1 68-71, ones2 72-75, zeros1 76-79, zeros2 80-82 and 73.  73 is
        // both ones2_i32 and zeros2_f64 (bytecode/ByteCodes.hpp:95-105); the
        // reference dispatches it as zeros2_f64, and so does this back end.
        n.kind = Node::FILL;
        int k, two, one;
        if (op == 73) { k = 3; two = 1; one = 0; }
        else if (op <= 71) { k = op - 68; two = 0; one = 1; }
        else if (op <= 75) { k = op - 72; two = 1; one = 1; }
        else if (op <= 79) { k = op - 76; two = 0; one = 0; }
        else { k = op - 80; two = 1; one = 0; }
        n.W = (uint64_t)scalar_cell(s, pos, ok);
        n.H = two ? (uint64_t)scalar_cell(s, pos, ok) : 1;
        n.scalar = one ? 1.0 : 0.0;
        n.prec = k == 0 ? CHAI_U32 : k == 1 ? CHAI_I32 : k == 2 ? CHAI_F32 : CHAI_F64;
        return ok ? add(n) : -1;
    }
    if (op >= 90 && op <= 101) {
        n.kind = Node::READ;
        int k = parse(s, pos);
        if (k < 0 || pos < 0 || s.cells[pos].kind != CHAI_BC_MEMORY) return -1;
        n.buffer = s.cells[pos--].buffer;
        n.kids = {k};
        n.read_kind = op <= 93 ? 0 : (op <= 97 ? 1 : 2);
        n.prec = nodes_[k].prec;
        n.W = nodes_[k].W; n.H = nodes_[k].H; n.slots = nodes_[k].slots;
        return add(n);
    }
    if (op == 50) {
        // kernel_from_opencl: [{KERNEL, index}, 50]
        if (pos < 0 || s.cells[pos].kind != CHAI_BC_KERNEL) return -1;
        const uint64_t kidx = s.cells[pos--].buffer;
        if (!kernels_ || kidx >= n_kernels_) return -1;
        const chai_inline_kernel& kd = kernels_[kidx];
        if (!kd.source || !kd.name || (kd.n_args && !kd.args)) return -1;
        n.kind = Node::INLINE;
        n.buffer = kidx;
        for (uint32_t a = 0; a < kd.n_args; a++) {
            if (kd.args[a].kind != CHAI_KARG_ARRAY) continue;
            Node v;
            v.kind = Node::VAR;
            v.var = kd.args[a].variable;
            v.ver = kd.args[a].version;
            int k = resolve_var(v);
            if (k < 0) return -1;
            // the kernel updates this argument in place: when its value is
            // also another variable's (equal expressions share one node) or
            // another argument of this kernel, the argument gets a private
            // copy, so that only this variable sees the update -- as every
            // chai array has memory of its own in the reference
            bool shared = std::find(n.kids.begin(), n.kids.end(), k) != n.kids.end();
            for (const auto& kv : assigned_)
                if (!shared && kv.second == k && kv.first.first != v.var) shared = true;
            for (const auto& kv : inputs_)
                if (!shared && kv.second == k && kv.first != v.var) shared = true;
            if (shared) {
                Node c;
                c.kind = Node::CONVERT;           // same precision: a copy
                c.prec = nodes_[k].prec;
                c.W = nodes_[k].W; c.H = nodes_[k].H; c.slots = nodes_[k].slots;
                c.kids = {k};
                c.var = v.var;                    // one copy per (variable, version)
                c.ver = v.ver;
                k = add(c);
            }
            n.kids.push_back(k);
        }
        return add(n);
    }
    if (op >= 110 && op <= 115) {
        n.kind = Node::RNG;
        n.variant = (uint32_t)scalar_cell(s, pos, ok);
        n.seed = (uint64_t)scalar_cell(s, pos, ok);
        n.W = (uint64_t)scalar_cell(s, pos, ok);
        n.H = (uint64_t)scalar_cell(s, pos, ok);
        n.slots = (uint32_t)scalar_cell(s, pos, ok);
        n.dist = (op == 110 || op == 111) ? 1 : 0;
        n.prec = (op == 110 || op == 114) ? CHAI_F32 : (op == 111 || op == 115) ? CHAI_F64
                 : op == 112 ? CHAI_U32 : CHAI_I32;
        if (op == 114 || op == 115) {
            n.lo = scalar_cell(s, pos, ok);
            n.hi = scalar_cell(s, pos, ok);
            n.limits = true;
        }
        if (n.variant != CHAI_RNG_PHILOX && n.variant != CHAI_RNG_THREEFRY) return -1;
        return ok ? add(n) : -1;
    }
    if (op == 120 || op == 121) {
        n.kind = op == 120 ? Node::MATMUL : Node::MATMULG;
        int a = parse(s, pos), b = parse(s, pos);
        if (a < 0 || b < 0) return -1;
        n.kids = {a, b};
        n.prec = wider(nodes_[a].prec, nodes_[b].prec);
        const Node& l = nodes_[a];
        const Node& r = nodes_[b];
        n.slots = std::max(l.slots, r.slots);
        if (op == 121) {
            int cc = parse(s, pos);
            if (cc < 0) return -1;
            n.kids.push_back(cc);
            n.alpha = scalar_cell(s, pos, ok);
            n.beta = scalar_cell(s, pos, ok);
            n.W = nodes_[cc].W; n.H = nodes_[cc].H;
            n.prec = wider(n.prec, nodes_[cc].prec);
            return ok ? add(n) : -1;
        }
        // api/ArrayFun.cpp:74-90
        if (l.H == 1 && r.H == 1) { n.W = r.W; n.H = l.W; }
        else if (l.H == 1) { n.W = r.W; n.H = 1; }
        else if (r.H == 1) { n.W = l.H; n.H = 1; }
        else { n.W = r.W; n.H = l.H; }
        return add(n);
    }
    if (op == 122) {
        n.kind = Node::TRANSPOSE;
        int a = parse(s, pos);
        if (a < 0) return -1;
        n.kids = {a};
        n.prec = nodes_[a].prec;
        n.W = nodes_[a].H; n.H = nodes_[a].W; n.slots = nodes_[a].slots;
        return add(n);
    }
    if (op >= 130 && op <= 132) {
        n.kind = Node::REDUCE;
        int a = parse(s, pos);
        if (a < 0) return -1;
        n.kids = {a};
        if (op == 130) {
            int b = parse(s, pos);
            if (b < 0) return -1;
            n.kids.push_back(b);
        }
        n.prec = nodes_[a].prec;
        for (int k : n.kids) n.prec = wider(n.prec, nodes_[k].prec);
        n.W = 1; n.H = 1;
        n.slots = nodes_[a].slots;
        return add(n);
    }
    const int ar = arity_of(op);
    if (ar < 0) {
        unsupported_op_ = op;
        return -1;
    }
    n.kind = (op == 40 || op == 41) ? Node::GATHER : Node::OP;
    for (int i = 0; i < ar; i++) {
        int k = parse(s, pos);
        if (k < 0) return -1;
        n.kids.push_back(k);
    }
    if (n.kind == Node::GATHER) {
        // FIRST2 / FIRST3: shape of the gathered array (api/ArrayFun.cpp:92-111)
        const Node& a = nodes_[n.kids[0]];
        n.W = a.W; n.H = a.H; n.slots = a.slots; n.prec = a.prec;
        for (size_t i = 1; i < n.kids.size(); i++) n.slots = std::max(n.slots, nodes_[n.kids[i]].slots);
        return add(n);
    }
    int p = 0;
    uint64_t W = 1, H = 1;
    uint32_t sl = 1;
    // cond(pred, a, b): precision of a and b only
    for (size_t i = (op == 23 ? 1 : 0); i < n.kids.size(); i++) p = wider(p, nodes_[n.kids[i]].prec);
    for (int k : n.kids) {
        W = std::max(W, nodes_[k].W);
        H = std::max(H, nodes_[k].H);
        sl = std::max(sl, nodes_[k].slots);
    }
    if (fp_only(op) && p < CHAI_F32) p = CHAI_F32;
    if (is_int_only(op) && p >= CHAI_F32) {
        unsupported_op_ = op;
        return -1;
    }
    n.prec = p;
    n.W = W; n.H = H; n.slots = sl;
    return add(n);
}

int Translator::resolve_var(const Node& v)
{
    // latest in-trace assignment of (variable, version)
    auto it = assigned_.find(std::make_pair(v.var, v.ver));
    if (it != assigned_.end()) return it->second;
    auto lit = latest_.find(v.var);
    if (lit != latest_.end()) return lit->second;
    // a bound input
    auto b = bindings_.find(v.var);
    if (b == bindings_.end()) return -1;
    auto in = inputs_.find(v.var);
    if (in != inputs_.end()) return in->second;
    Node n;
    n.kind = Node::INPUT;
    n.var = v.var;
    n.prec = (int)b->second.prec;
    n.W = b->second.width; n.H = b->second.height; n.slots = b->second.slots;
    n.buffer = b->second.buffer;
    int id = add(n);
    inputs_[v.var] = id;
    return id;
}

// ----------------------------------------------------------- evaluate

int Translator::parse_only(const chai_trace_desc* t)
{
    slots_ = t->num_traces ? t->num_traces : 1;
    for (uint32_t i = 0; i < t->n_stmts; i++) {
        const chai_stmt& s = t->stmts[i];
        if (!s.cells || s.n_cells == 0) return fail(CHAI_ERR_INVALID, "empty statement");
        int pos = (int)s.n_cells - 1;
        const int root = parse(s, pos);
        if (root < 0 || pos != -1) return fail(CHAI_ERR_INVALID, "malformed statement");
        if (nodes_[root].kind == Node::READ) {
            reads_.push_back(root);
        } else {
            assigned_[std::make_pair(s.lhs_variable, s.lhs_version)] = root;
            latest_[s.lhs_variable] = root;
            stmt_roots_.push_back(std::make_pair(s.lhs_variable, root));
        }
    }
    return CHAI_OK;
}

int Translator::result_root() const
{
    if (stmt_roots_.empty()) return -1;
    const int r = stmt_roots_.back().second;
    return nodes_[r].kind == Node::REDUCE ? r : -1;
}

int Translator::read_result(double* out)
{
    const int r = result_root();
    if (r < 0 || !nodes_[r].dev) return fail(CHAI_ERR_UNSUPPORTED, "trace has no reduction result");
    const Node& n = nodes_[r];
    unsigned char buf[8] = {0};
    CHAI_CUDA_TRY(ctx_, cudaMemcpyAsync(buf, n.dev, prec_bytes(n.prec), cudaMemcpyDeviceToHost, ctx_->stream));
    CHAI_CUDA_TRY(ctx_, cudaStreamSynchronize(ctx_->stream));
    switch (n.prec) {
        case CHAI_F32: { float v; memcpy(&v, buf, 4); *out = v; break; }
        case CHAI_F64: { double v; memcpy(&v, buf, 8); *out = v; break; }
        case CHAI_I32: { int v; memcpy(&v, buf, 4); *out = v; break; }
        default: { unsigned v; memcpy(&v, buf, 4); *out = v; break; }
    }
    return CHAI_OK;
}

// Steps 1-2 of a run: parse every statement into the node DAG, with the
// bindings (input shapes) and inline kernels of the trace.
int Translator::parse_all(const chai_trace_desc* t, const chai_buffer_binding* binds, size_t nb)
{
    for (size_t i = 0; i < nb; i++) bindings_[binds[i].variable] = binds[i];
    slots_ = t->num_traces ? t->num_traces : 1;
    kernels_ = t->kernels;
    n_kernels_ = t->kernels ? t->n_kernels : 0;
    first_inline_ = -1;
    for (uint32_t i = 0; i < t->n_stmts; i++) {
        const chai_stmt& s = t->stmts[i];
        if (!s.cells || s.n_cells == 0) return fail(CHAI_ERR_INVALID, "empty statement");
        int pos = (int)s.n_cells - 1;
        int root = parse(s, pos);
        if (root < 0) {
            if (unsupported_op_)
                return fail(CHAI_ERR_UNSUPPORTED, "unsupported opcode " + std::to_string(unsupported_op_));
            return fail(CHAI_ERR_INVALID, "malformed statement " + std::to_string(i));
        }
        if (pos != -1) return fail(CHAI_ERR_INVALID, "trailing cells in statement " + std::to_string(i));
        if (nodes_[root].kind == Node::READ) {
            reads_.push_back(root);
        } else if (nodes_[root].kind == Node::INLINE) {
            // the kernel updates its array arguments in place: later statements
            // reading (variable, version) see the values after the kernel
            if (first_inline_ < 0) first_inline_ = (int)stmt_roots_.size();
            stmt_roots_.push_back(std::make_pair(s.lhs_variable, root));
            const chai_inline_kernel& kd = kernels_[nodes_[root].buffer];
            size_t m = 0;
            for (uint32_t a = 0; a < kd.n_args; a++) {
                if (kd.args[a].kind != CHAI_KARG_ARRAY) continue;
                const int pre = nodes_[root].kids[m++];
                Node after;
                after.kind = Node::AFTER;
                after.kids = {root, pre};
                after.prec = nodes_[pre].prec;
                after.W = nodes_[pre].W; after.H = nodes_[pre].H; after.slots = nodes_[pre].slots;
                after.var = kd.args[a].variable;
                after.ver = kd.args[a].version;
                const int id = add(after);
                assigned_[std::make_pair(kd.args[a].variable, kd.args[a].version)] = id;
                latest_[kd.args[a].variable] = id;
            }
        } else {
            assigned_[std::make_pair(s.lhs_variable, s.lhs_version)] = root;
            latest_[s.lhs_variable] = root;
            stmt_roots_.push_back(std::make_pair(s.lhs_variable, root));
            stmt_values_.push_back({s.lhs_variable, s.lhs_version, (uint32_t)nodes_[root].prec,
                                    nodes_[root].slots, nodes_[root].W, nodes_[root].H});
        }
    }
    return CHAI_OK;
}

int Translator::run(const chai_trace_desc* t, const chai_buffer_binding* binds, size_t nb)
{
    int pst = parse_all(t, binds, nb);
    if (pst) return pst;
    const int first_inline = first_inline_;      // statement index of the first inline kernel
    // 3: materialisation
    materialize_.assign(nodes_.size(), false);
    for (size_t i = 0; i < nodes_.size(); i++) {
        const Node& n = nodes_[i];
        switch (n.kind) {
            case Node::MATMUL: case Node::MATMULG: case Node::TRANSPOSE:
                materialize_[i] = true;
                for (int k : n.kids) materialize_[k] = true;
                break;
            case Node::REDUCE:
                materialize_[i] = true;
                break;
            case Node::GATHER:
                materialize_[n.kids[0]] = true;
                break;
            case Node::READ:
                materialize_[n.kids[0]] = true;
                break;
            case Node::INPUT:
            case Node::MAKE:
                materialize_[i] = true;   // values that already live in HBM
                break;
            case Node::INLINE:
                materialize_[i] = true;
                for (int k : n.kids) materialize_[k] = true;
                break;
            case Node::AFTER:
                materialize_[i] = true;
                break;
            default:
                break;
        }
    }
    for (auto& kv : latest_)
        if (bindings_.count(kv.first)) materialize_[kv.second] = true;
    // an inline kernel is a barrier: every value assigned before it is
    // computed (into HBM) before it runs
    for (int k = 0; k < first_inline; k++) {
        const int r = stmt_roots_[k].second;
        if (nodes_[r].kind != Node::INLINE) materialize_[r] = true;
    }
    // storage for materialised nodes
    for (size_t i = 0; i < nodes_.size(); i++) {
        if (!materialize_[i]) continue;
        int st = assign_storage((int)i);
        if (st) return st;
    }
    // 4-5: group and launch in statement order
    std::vector<int> order;
    std::vector<bool> seen(nodes_.size(), false);
    std::function<void(int)> visit = [&](int i) {
        if (seen[i]) return;
        seen[i] = true;
        for (int k : nodes_[i].kids) visit(k);
        if (materialize_[i]) order.push_back(i);
    };
    for (auto& sr : stmt_roots_) visit(sr.second);
    for (int r : reads_) visit(r);
    int st = schedule(order);
    if (st) return st;
    if (dry_) return CHAI_OK;
    // read-backs into the FrontMem stand-in buffers
    for (int r : reads_) {
        st = do_read(r);
        if (st) return st;
    }
    // bound outputs that alias a different node (plain `a = b` statements)
    for (auto& kv : latest_) {
        auto b = bindings_.find(kv.first);
        if (b == bindings_.end()) continue;
        const Node& n = nodes_[kv.second];
        if (n.kind == Node::INPUT && n.var == kv.first) continue;
        if (n.storage_buffer == b->second.buffer) continue;
        // (a value updated in place by an inline kernel lives in its
        // argument's storage; the bound buffer may not exist yet)
        int ast = alloc_buffer(ctx_, b->second.buffer, node_bytes(n));
        if (ast) return ast;
        Buffer* dst = find_buffer(ctx_, b->second.buffer);
        if (!dst) return fail(CHAI_ERR_NOT_FOUND, "output buffer");
        note_buffer(b->second.buffer, node_bytes(n), true);
        Step cs;
        cs.kind = Step::COPY;
        cs.a = ref_of(dst->ptr);
        cs.b = ref_of(n.dev);
        cs.bytes = node_bytes(n);
        int st = exec(cs);
        if (st) return st;
    }
    return CHAI_OK;
}

size_t Translator::node_bytes(const Node& n) const
{
    return (size_t)n.W * n.H * n.slots * prec_bytes(n.prec);
}

int Translator::assign_storage(int i)
{
    Node& n = nodes_[i];
    if (n.dev) return CHAI_OK;
    if (n.kind == Node::INLINE) return CHAI_OK;       // no value of its own
    if (n.kind == Node::AFTER) {                       // the argument's storage, updated in place
        const Node& pre = nodes_[n.kids[1]];
        n.dev = pre.dev;
        n.storage_buffer = pre.storage_buffer;
        return CHAI_OK;
    }
    if (dry_) {
        n.dev = reinterpret_cast<void*>(uintptr_t(0x10000) * (i + 1));
        return CHAI_OK;
    }
    if (n.kind == Node::INPUT || n.kind == Node::MAKE) {
        Buffer* b = find_buffer(ctx_, n.buffer);
        if (!b) return fail(CHAI_ERR_NOT_FOUND, "input buffer " + std::to_string(n.buffer));
        if (b->bytes < node_bytes(n)) return fail(CHAI_ERR_INVALID, "input buffer too small");
        n.dev = b->ptr;
        n.storage_buffer = n.buffer;
        note_buffer(n.buffer, node_bytes(n), false);
        return CHAI_OK;
    }
    // the node is the final value of a bound variable -> its buffer.  Not when
    // that variable is also an input of this trace: its buffer then holds the
    // input, which a GEMM, a gather or a later kernel of this trace may still
    // read, so the value goes to a temporary and is copied into the buffer
    // after the last kernel (run(), bound outputs that alias another node).
    for (auto& kv : latest_) {
        if (kv.second != i) continue;
        auto b = bindings_.find(kv.first);
        if (b == bindings_.end()) continue;
        if (inputs_.count(kv.first)) break;
        int st = alloc_buffer(ctx_, b->second.buffer, node_bytes(n));
        if (st) return st;
        note_buffer(b->second.buffer, node_bytes(n), true);
        Buffer* buf = find_buffer(ctx_, b->second.buffer);
        n.dev = buf->ptr;
        n.storage_buffer = b->second.buffer;
        return CHAI_OK;
    }
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(256, (node_bytes(n) + 255) & ~size_t(255));
    CHAI_CUDA_TRY(ctx_, cudaMallocAsync(&p, bytes, ctx_->stream));
    temps_.push_back(p);
    temp_sizes_.push_back(bytes);
    n.dev = p;
    return CHAI_OK;
}

Translator::~Translator()
{
    for (void* p : temps_) cudaFreeAsync(p, ctx_->stream);
}

// Group consecutive element roots with one iteration space into one kernel.
int Translator::schedule(const std::vector<int>& order)
{
    std::vector<int> group;
    std::set<int> in_group;
    uint64_t gW = 0, gH = 0;
    uint32_t gS = 0;
    auto flush = [&]() -> int {
        if (group.empty()) return CHAI_OK;
        int st = emit_group(group);
        group.clear();
        in_group.clear();
        return st;
    };
    // does node i (transitively, through register values) need a complete
    // in-group result: a gather source or a reduction computed in the group?
    std::function<bool(int, std::set<int>&)> needs_barrier = [&](int i, std::set<int>& vis) -> bool {
        if (vis.count(i)) return false;
        vis.insert(i);
        const Node& n = nodes_[i];
        if (n.kind == Node::GATHER && in_group.count(n.kids[0])) return true;
        for (int k : n.kids) {
            if (in_group.count(k) && nodes_[k].kind == Node::REDUCE) return true;
            if (materialize_[k] && !in_group.count(k)) continue;
            if (needs_barrier(k, vis)) return true;
        }
        return false;
    };
    for (int i : order) {
        Node& n = nodes_[i];
        if (n.kind == Node::INPUT || n.kind == Node::MAKE || n.kind == Node::AFTER) continue;
        if (n.kind == Node::INLINE) {
            int st = flush();
            if (st) return st;
            st = emit_inline(i);
            if (st) return st;
            continue;
        }
        if (n.kind == Node::MATMUL || n.kind == Node::MATMULG || n.kind == Node::TRANSPOSE) {
            int st = flush();
            if (st) return st;
            st = emit_linalg(i);
            if (st) return st;
            continue;
        }
        // iteration space: the reduction's operand, else the node itself
        uint64_t W = n.W, H = n.H;
        uint32_t S = n.slots;
        if (n.kind == Node::REDUCE) {
            W = 1; H = 1;
            for (int k : n.kids) {
                W = std::max(W, nodes_[k].W);
                H = std::max(H, nodes_[k].H);
            }
        }
        std::set<int> vis;
        const bool same = !group.empty() && W == gW && H == gH && S == gS;
        if (!same || needs_barrier(i, vis)) {
            int st = flush();
            if (st) return st;
            gW = W; gH = H; gS = S;
        }
        group.push_back(i);
        in_group.insert(i);
    }
    return flush();
}

}  // namespace chai
