// Many traces of uneven length in one persistent launch, replayed from a
// captured CUDA graph (chai_cuda_evaluate_many).
//
// The reference batches only traces with the same hash (runtime/Scheduler.cpp:
// 48-89), and the hash covers W and H, so traces of different lengths each get
// their own dispatch; a VectorTrace also needs equal slot shapes
// (api/chai.h:551-600).  Here traces that share one program -- the same cells
// except for scalar values (W, H, seeds, literals) -- are compiled once, with
// the per-trace scalars read from a device table, and run as ONE kernel over a
// global list of 4096-element tiles (256 threads x 4 chunks of 4; small
// enough that the last of ~15 tiles per CTA leaves little of the grid idle):
//   tab[0] = number of tiles, tab[1] = number of traces, then per trace:
//   { n, W, H, first tile, seed of each RNG node, bits of each varying scalar }.
// Every CTA walks a contiguous run of tiles (equal runs to within one tile);
// its first tile finds its trace by binary search on the first-tile column
// and later tiles follow the column; a CTA keeps its running sum over
// consecutive tiles of one trace in registers and writes its block partial at
// its last tile of that trace (0 for the others) to partials[tile]; a second
// kernel adds each trace's partials in tile order in FP64.  The H2D copy of the table, both kernels and the D2H copy of the
// results are captured once into a CUDA graph per (program, trace count) and
// replayed afterwards.
//
// Scope: traces made only of element operations (literals, index arrays,
// Random123 arrays, unary / binary / ternary ops, conversions) of the
// iteration's shape, with W and n multiples of 4, ending in one reduction whose
// value is the trace's result.  Other traces are evaluated one by one through
// chai_cuda_evaluate (same results, one dispatch each).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cinttypes>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <vector>

#include "internal.h"
#include "jit.h"
#include "trace.h"

namespace chai {

constexpr int kManySubs = 4;                       // chunks of 4 elements per thread and tile
constexpr long long kManyTile = 256 * 4 * kManySubs;

int launch_many_combine(chai_cuda_ctx* ctx, const long long* tab, int stride, const double* partials, double* out,
                        int ntr, int mean, int prec);

namespace {

const char* ctype_m(int prec)
{
    switch (prec) {
        case CHAI_U32: return "unsigned";
        case CHAI_I32: return "int";
        case CHAI_F32: return "float";
        case CHAI_F64: return "double";
    }
    return "float";
}

struct ManyGraph {
    cudaGraphExec_t exec = nullptr;
    long long* dev_tab = nullptr;
    long long* host_tab = nullptr;     // pinned
    double* dev_res = nullptr;
    double* host_res = nullptr;        // pinned
    double* partials = nullptr;
    long long cap_tiles = 0;
    size_t tab_words = 0;
};

// Per-context state lives in maps keyed by the context; the lock covers
// finding or inserting a context's entry (contexts may be driven from
// different threads), after which only that context's thread touches it.
std::mutex g_many_mu;

std::map<std::pair<uint64_t, size_t>, ManyGraph>& graphs(chai_cuda_ctx* ctx)
{
    static std::map<chai_cuda_ctx*, std::map<std::pair<uint64_t, size_t>, ManyGraph>> all;
    std::lock_guard<std::mutex> g(g_many_mu);
    return all[ctx];
}

}  // namespace

// Free the graphs and buffers of a context (chai_cuda_shutdown).
void clear_last_batch(chai_cuda_ctx* ctx);

void many_release(chai_cuda_ctx* ctx)
{
    auto& m = graphs(ctx);
    for (auto& kv : m) {
        ManyGraph& g = kv.second;
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.dev_tab) cudaFree(g.dev_tab);
        if (g.host_tab) cudaFreeHost(g.host_tab);
        if (g.dev_res) cudaFree(g.dev_res);
        if (g.host_res) cudaFreeHost(g.host_res);
        if (g.partials) cudaFree(g.partials);
    }
    m.clear();
    clear_last_batch(ctx);
}

// Program description shared by all traces (built from trace 0).
struct ManyProgram {
    std::string source;
    int stride = 0;                 // table words per trace
    std::vector<int> rng_nodes;     // table column 4 + k
    std::vector<int> var_scalars;   // table column 4 + nrng + k
    int red_op = 132, red_prec = CHAI_F32;
};

// The last persistent batch of a context: its traces' statements and cells
// (scalars included) byte for byte, and what parsing them produced.  A call
// whose batch repeats it skips parsing, program generation and the table
// build, and goes straight to the captured graph.
struct ManyLast {
    bool valid = false;
    std::string content;
    ManyProgram prog;
    std::vector<long long> tab;
    void* fn = nullptr;
    uint64_t key = 0;
};

ManyLast& last_batch(chai_cuda_ctx* ctx)
{
    static std::map<chai_cuda_ctx*, ManyLast> all;
    std::lock_guard<std::mutex> g(g_many_mu);
    return all[ctx];
}

void clear_last_batch(chai_cuda_ctx* ctx) { last_batch(ctx) = ManyLast(); }

// Statements and cells of a batch as bytes; false for batches with inline
// kernels (their program text is not part of the statements).
bool batch_content(const chai_trace_desc* const* traces, size_t n, std::string& out)
{
    out.clear();
    auto put = [&](const void* p, size_t b) { out.append(static_cast<const char*>(p), b); };
    for (size_t t = 0; t < n; t++) {
        const chai_trace_desc* d = traces[t];
        if (!d || d->n_kernels || (d->n_stmts && !d->stmts)) return false;
        put(&d->num_traces, 4);
        put(&d->n_stmts, 4);
        for (uint32_t i = 0; i < d->n_stmts; i++) {
            const chai_stmt& st = d->stmts[i];
            if (st.n_cells && !st.cells) return false;
            put(&st.lhs_variable, 4);
            put(&st.lhs_version, 4);
            put(&st.n_cells, 4);
            for (uint32_t c = 0; c < st.n_cells; c++) {
                const chai_bc& b = st.cells[c];
                put(&b.kind, 4);
                put(&b.code, 4);
                put(&b.version, 4);
                put(&b.scalar, 8);
                put(&b.buffer, 8);
            }
        }
    }
    return true;
}

static bool same_structure(const std::vector<Node>& a, const std::vector<Node>& b)
{
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); i++)
        if (a[i].kind != b[i].kind || a[i].op != b[i].op || a[i].prec != b[i].prec || a[i].kids != b[i].kids ||
            a[i].variant != b[i].variant || a[i].dist != b[i].dist || a[i].limits != b[i].limits ||
            a[i].dim != b[i].dim)
            return false;
    return true;
}

// Codegen of the multi-trace kernel; false when the program is out of scope.
static bool build_program(const std::vector<std::vector<Node>>& all, int root, double two_pi, int layout,
                          ManyProgram& p)
{
    const std::vector<Node>& nodes = all[0];
    const Node& red = nodes[root];
    if (red.kind != Node::REDUCE || red.kids.size() != 1) return false;
    p.red_op = (int)red.op;
    p.red_prec = red.prec;
    // body: every node reachable from the reduction operand
    std::vector<int> body;
    std::set<int> seen;
    std::function<bool(int)> dfs = [&](int i) -> bool {
        if (seen.count(i)) return true;
        seen.insert(i);
        const Node& n = nodes[i];
        switch (n.kind) {
            case Node::SCALAR: case Node::FILL: case Node::CONVERT: case Node::INDEX: case Node::OP: case Node::RNG:
                break;
            default:
                return false;
        }
        for (int k : n.kids)
            if (!dfs(k)) return false;
        body.push_back(i);
        return true;
    };
    if (!dfs(red.kids[0])) return false;
    const int it = red.kids[0];
    for (const auto& tr : all) {
        const Node& r = tr[it];
        if ((r.W * r.H) % 4 != 0 || r.W % 4 != 0 || r.slots != 1) return false;
        for (int i : body) {
            const Node& n = tr[i];
            if ((n.kind == Node::RNG || n.kind == Node::INDEX) && (n.W != r.W || n.H != r.H || n.slots != 1))
                return false;
            if (n.kind != Node::SCALAR && n.kind != Node::FILL && n.kind != Node::RNG && (n.W != r.W || n.H != r.H) &&
                !(n.W == 1 && n.H == 1))
                return false;
        }
    }
    // varying scalars
    for (int i : body) {
        const Node& n = nodes[i];
        if (n.kind == Node::RNG) p.rng_nodes.push_back(i);
        if (n.kind == Node::SCALAR) {
            for (const auto& tr : all)
                if (memcmp(&tr[i].scalar, &n.scalar, 8) != 0) {
                    p.var_scalars.push_back(i);
                    break;
                }
        }
    }
    p.stride = 4 + (int)p.rng_nodes.size() + (int)p.var_scalars.size();
    auto col_of = [&](const std::vector<int>& v, int i) { return (int)(std::find(v.begin(), v.end(), i) - v.begin()); };
    // element indices in 32 bits when every trace is shorter than 2^30
    // elements (the chunk index c = e0 / 4 and its bound then fit an int)
    bool small = true;
    for (const auto& tr : all) small = small && (long long)(tr[it].W * tr[it].H) < (1ll << 30);
    std::ostringstream os;
    os << "extern \"C\" __global__ void __launch_bounds__(256) chai_many(const long long* __restrict__ tab, "
          "double* __restrict__ partials)\n{\n  using namespace chai_ops; using namespace chai_rng;\n"
       << "  const long long ntiles = tab[0]; const int ntr = (int)tab[1];\n"
       << "  const long long* rows = tab + 2;\n"
       << "  double red[1] = {0};\n"
       // each CTA takes a contiguous run of tiles, so consecutive tiles mostly
       // share a trace (one reduction per trace and CTA); the trace is found
       // by binary search at the run's first tile and followed from there
       << "  const long long t0 = ntiles * blockIdx.x / gridDim.x, t1 = ntiles * (blockIdx.x + 1) / gridDim.x;\n"
       << "  int lo = 0;\n"
       << "  { int hi = ntr - 1; while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (rows[(long long)mid * "
       << p.stride << " + 3] <= t0) lo = mid; else hi = mid - 1; } }\n"
       << "  for (long long tile = t0; tile < t1; tile++) {\n"
       << "    while (lo + 1 < ntr && rows[(long long)(lo + 1) * " << p.stride << " + 3] <= tile) lo++;\n"
       << "    const long long* tp = rows + (long long)lo * " << p.stride << ";\n"
       << "    const long long n = tp[0], W = tp[1];\n"
       << "    const long long next = tile + 1;\n"
       << "    const bool flush = next >= t1 || (lo + 1 < ntr && rows[(long long)(lo + 1) * " << p.stride
       << " + 3] <= next);\n"
       << "    for (int sub = 0; sub < " << kManySubs << "; sub++) {\n"
       << (small ? "    const int c = ((int)(tile - tp[3]) * " : "    const long long c = ((tile - tp[3]) * ") << kManySubs
       << " + sub) * 256 + threadIdx.x;\n"
       << (small ? "    if (c * 4 >= (int)n) break;\n" : "    if (c * 4 >= n) break;\n")
       << "    const long long e0 = (long long)c * 4;\n"
       << "    long long xx[4], yy[4]; { const long long y0 = e0 / W, x0 = e0 - y0 * W; "
          "for (int j = 0; j < 4; j++) { xx[j] = x0 + j; yy[j] = y0; } }\n";
    for (int i : body) {
        const Node& nd = nodes[i];
        const char* T = ctype_m(nd.prec);
        os << "    " << T << " v" << i << "[4];\n";
        switch (nd.kind) {
            case Node::SCALAR:
            case Node::FILL: {
                const int col = col_of(p.var_scalars, i);
                if (nd.kind == Node::SCALAR && col < (int)p.var_scalars.size())
                    os << "    { const double t = __longlong_as_double(tp[" << 4 + p.rng_nodes.size() + col
                       << "]); for (int j = 0; j < 4; j++) v" << i << "[j] = (" << T << ")t; }\n";
                else {
                    double v = nd.scalar;
                    uint64_t u;
                    memcpy(&u, &v, 8);
                    char buf[64];
                    snprintf(buf, sizeof buf, "__longlong_as_double(0x%016" PRIx64 "ull)", u);
                    os << "    for (int j = 0; j < 4; j++) v" << i << "[j] = (" << T << ")" << buf << ";\n";
                }
                break;
            }
            case Node::CONVERT:
                os << "    for (int j = 0; j < 4; j++) v" << i << "[j] = (" << T << ")v" << nd.kids[0] << "[j];\n";
                break;
            case Node::INDEX:
                os << "    for (int j = 0; j < 4; j++) v" << i << "[j] = (" << T << ")" << (nd.dim == 0 ? "xx" : "yy")
                   << "[j];\n";
                break;
            case Node::OP: {
                const int ar = (int)nd.kids.size();
                if (nd.op == 23) {
                    os << "    for (int j = 0; j < 4; j++) v" << i << "[j] = (v" << nd.kids[0] << "[j] != 0) ? (" << T
                       << ")v" << nd.kids[1] << "[j] : (" << T << ")v" << nd.kids[2] << "[j];\n";
                    break;
                }
                os << "    for (int j = 0; j < 4; j++) v" << i << "[j] = f" << ar << "<" << nd.op << ", " << T << ">(";
                for (int k = 0; k < ar; k++) os << (k ? ", " : "") << "(" << T << ")v" << nd.kids[k] << "[j]";
                os << ");\n";
                break;
            }
            case Node::RNG: {
                const int col = 4 + col_of(p.rng_nodes, i);
                const std::string tmpl = "<" + std::to_string(nd.variant) + ", " + std::to_string(layout) + ">";
                char tp[64];
                snprintf(tp, sizeof tp, "__int_as_float(0x%08x)", [&] { float f = (float)two_pi; uint32_t u; memcpy(&u, &f, 4); return u; }());
                if (nd.prec == CHAI_F64) {
                    char tp64[64];
                    uint64_t u;
                    memcpy(&u, &two_pi, 8);
                    snprintf(tp64, sizeof tp64, "__longlong_as_double(0x%016" PRIx64 "ull)", u);
                    os << "    for (int h = 0; h < 2; h++) { const u64x2 r = raw64" << tmpl
                       << "((unsigned long long)(e0 >> 1) + h, (unsigned long long)tp[" << col << "]);\n";
                    if (nd.dist == 1)
                        os << "      box_muller_f64(u01_f64(r.x), u01_f64(r.y), " << tp64 << ", v" << i << "[2 * h], v" << i
                           << "[2 * h + 1]); }\n";
                    else
                        os << "      v" << i << "[2 * h] = u01_f64(r.x); v" << i << "[2 * h + 1] = u01_f64(r.y); }\n";
                } else {
                    os << "    { const u32x4 r = raw32" << tmpl << "((unsigned)(e0 >> 2), (unsigned)tp[" << col
                       << "], true);\n";
                    if (nd.dist == 1) {
                        os << "      box_muller_f32(u01_f32(r.x), u01_f32(r.y), " << tp << ", v" << i << "[0], v" << i
                           << "[1]);\n      box_muller_f32(u01_f32(r.z), u01_f32(r.w), " << tp << ", v" << i << "[2], v"
                           << i << "[3]);\n";
                    } else if (nd.prec == CHAI_F32) {
                        os << "      v" << i << "[0] = u01_f32(r.x); v" << i << "[1] = u01_f32(r.y); v" << i
                           << "[2] = u01_f32(r.z); v" << i << "[3] = u01_f32(r.w);\n";
                    } else {
                        os << "      v" << i << "[0] = (" << T << ")r.x; v" << i << "[1] = (" << T << ")r.y; v" << i
                           << "[2] = (" << T << ")r.z; v" << i << "[3] = (" << T << ")r.w;\n";
                    }
                    os << "    }\n";
                }
                if (nd.limits && nd.dist == 0 && (nd.prec == CHAI_F32 || nd.prec == CHAI_F64)) {
                    if (nd.prec == CHAI_F32) {
                        const float len = (float)(nd.hi - nd.lo), lo = (float)nd.lo;
                        uint32_t ul, uo;
                        memcpy(&ul, &len, 4);
                        memcpy(&uo, &lo, 4);
                        os << "    for (int j = 0; j < 4; j++) { float t = __fmul_rn(v" << i << "[j], __int_as_float(0x"
                           << std::hex << ul << std::dec << "));";
                        if (nd.lo != 0.0) os << " t = __fadd_rn(t, __int_as_float(0x" << std::hex << uo << std::dec << "));";
                        os << " v" << i << "[j] = t; }\n";
                    } else {
                        const double len = nd.hi - nd.lo;
                        uint64_t ul, uo;
                        memcpy(&ul, &len, 8);
                        memcpy(&uo, &nd.lo, 8);
                        os << "    for (int j = 0; j < 4; j++) { double t = __dmul_rn(v" << i
                           << "[j], __longlong_as_double(0x" << std::hex << ul << std::dec << "ull));";
                        if (nd.lo != 0.0)
                            os << " t = __dadd_rn(t, __longlong_as_double(0x" << std::hex << uo << std::dec << "ull));";
                        os << " v" << i << "[j] = t; }\n";
                    }
                }
                break;
            }
            default:
                return false;
        }
    }
    // the CTA's running sum stays in registers over its tiles of one trace
    // and is reduced at its last tile of that trace; its other tiles of the
    // trace contribute 0 to the trace's partials (the combine adds all)
    os << "    for (int j = 0; j < 4; j++) red[0] += (double)v" << it << "[j];\n    }\n"
       << "    if (!flush) { if (threadIdx.x == 0) partials[tile] = 0.0; continue; }\n"
       << "    chai_k::block_sum<1, 256>(red);\n"
       << "    if (threadIdx.x == 0) partials[tile] = red[0];\n"
       << "    red[0] = 0;\n"
       << "    __syncthreads();\n  }\n}\n";
    p.source = os.str();
    return true;
}

}  // namespace chai

using namespace chai;

static int launch_batch(chai_cuda_ctx* ctx, ManyLast& b, size_t n_traces, double* results);

extern "C" int chai_cuda_evaluate_many(chai_cuda_ctx* ctx, const chai_trace_desc* const* traces, size_t n_traces,
                                       double* results)
{
    if (!ctx || (!traces && n_traces) || (!results && n_traces)) return CHAI_ERR_INVALID;
    if (n_traces == 0) return CHAI_OK;
    if (fault_injected("evaluate")) return set_error(ctx, CHAI_ERR_INJECTED, "injected evaluate failure");
    cudaSetDevice(ctx->device);
    std::string content;
    const bool cacheable = batch_content(traces, n_traces, content);
    ManyLast& last = last_batch(ctx);
    if (cacheable && last.valid && last.content == content)
        return launch_batch(ctx, last, n_traces, results);
    last.valid = false;
    // parse every trace (dry: no storage, no launches) to compare structures
    std::vector<std::vector<Node>> all;
    all.reserve(n_traces);
    int root = -1;
    bool persistent = true;
    for (size_t t = 0; t < n_traces && persistent; t++) {
        Translator tr(ctx, true);
        if (tr.parse_only(traces[t]) != CHAI_OK) { persistent = false; break; }
        all.push_back(tr.nodes());
        const int r = tr.result_root();
        if (t == 0) root = r;
        if (r < 0 || r != root || (t > 0 && !same_structure(all[0], all.back()))) persistent = false;
    }
    ManyProgram prog;
    if (persistent) persistent = build_program(all, root, 2.0 * ctx->cfg.rng_pi, ctx->cfg.rng_layout, prog);
    if (!persistent) {
        // one dispatch per trace through the regular translator
        for (size_t t = 0; t < n_traces; t++) {
            Translator tr(ctx);
            int st = tr.run(traces[t], nullptr, 0);
            if (st) return st;
            double v = 0;
            st = tr.read_result(&v);
            if (st) return st;
            results[t] = v;
        }
        return CHAI_OK;
    }
    void* fn = nullptr;
    int st = ctx->jit->get(prog.source, "chai_many", &fn);
    if (st) return st;
    // per-trace table
    const int it = all[0][root].kids[0];
    std::vector<long long> tab(2 + n_traces * prog.stride);
    long long tiles = 0;
    for (size_t t = 0; t < n_traces; t++) {
        long long* row = tab.data() + 2 + t * prog.stride;
        const Node& r = all[t][it];
        row[0] = (long long)(r.W * r.H);
        row[1] = (long long)r.W;
        row[2] = (long long)r.H;
        row[3] = tiles;
        tiles += (row[0] + kManyTile - 1) / kManyTile;
        for (size_t k = 0; k < prog.rng_nodes.size(); k++) {
            const Node& rn = all[t][prog.rng_nodes[k]];
            row[4 + k] = (long long)(rn.prec == CHAI_F64 ? rn.seed : (uint32_t)rn.seed);
        }
        for (size_t k = 0; k < prog.var_scalars.size(); k++)
            memcpy(&row[4 + prog.rng_nodes.size() + k], &all[t][prog.var_scalars[k]].scalar, 8);
    }
    tab[0] = tiles;
    tab[1] = (long long)n_traces;
    last.content.swap(content);
    last.prog = prog;
    last.tab.swap(tab);
    last.fn = fn;
    last.key = fnv1a64(prog.source.data(), prog.source.size());
    last.valid = cacheable;
    return launch_batch(ctx, last, n_traces, results);
}

// Run a parsed batch: upload its table through the (program, trace count)
// graph, capturing the graph first when there is none or it is too small.
static int launch_batch(chai_cuda_ctx* ctx, ManyLast& b, size_t n_traces, double* results)
{
    const ManyProgram& prog = b.prog;
    void* fn = b.fn;
    const std::vector<long long>& tab = b.tab;
    const long long tiles = tab[0];
    ManyGraph& g = graphs(ctx)[std::make_pair(b.key, n_traces)];
    const size_t words = tab.size();
    if (!g.exec || g.cap_tiles < tiles || g.tab_words != words) {
        // (re)build the buffers and the graph
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.dev_tab) cudaFree(g.dev_tab);
        if (g.host_tab) cudaFreeHost(g.host_tab);
        if (g.dev_res) cudaFree(g.dev_res);
        if (g.host_res) cudaFreeHost(g.host_res);
        if (g.partials) cudaFree(g.partials);
        g = ManyGraph();
        g.cap_tiles = std::max<long long>(tiles, 1024);
        g.tab_words = words;
        CHAI_CUDA_TRY(ctx, cudaMalloc(&g.dev_tab, words * sizeof(long long)));
        CHAI_CUDA_TRY(ctx, cudaMallocHost(&g.host_tab, words * sizeof(long long)));
        CHAI_CUDA_TRY(ctx, cudaMalloc(&g.dev_res, n_traces * sizeof(double)));
        CHAI_CUDA_TRY(ctx, cudaMallocHost(&g.host_res, n_traces * sizeof(double)));
        CHAI_CUDA_TRY(ctx, cudaMalloc(&g.partials, g.cap_tiles * sizeof(double)));
        memcpy(g.host_tab, tab.data(), words * sizeof(long long));
        cudaStream_t s = ctx->stream;
        cudaGraph_t graph;
        CHAI_CUDA_TRY(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaMemcpyAsync(g.dev_tab, g.host_tab, words * sizeof(long long), cudaMemcpyHostToDevice, s);
        const unsigned grid = (unsigned)(ctx->sm_count * 8);     // as the single-trace kernels
        void* args[2] = {&g.dev_tab, &g.partials};
        int lst = ctx->jit->launch(fn, dim3(grid), dim3(256), 0, args);
        int cst = launch_many_combine(ctx, g.dev_tab, prog.stride, g.partials, g.dev_res, (int)n_traces,
                                      prog.red_op == 131, prog.red_prec);
        cudaMemcpyAsync(g.host_res, g.dev_res, n_traces * sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (lst || cst || e != cudaSuccess) {
            if (e == cudaSuccess) cudaGraphDestroy(graph);
            return set_error(ctx, CHAI_ERR_LAUNCH, "evaluate_many: graph capture failed");
        }
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_status(ctx, e, "cudaGraphInstantiate");
    } else {
        memcpy(g.host_tab, tab.data(), words * sizeof(long long));
    }
    cudaEvent_t kev[2];
    ktime_begin(ctx, "many", kev);
    CHAI_CUDA_TRY(ctx, cudaGraphLaunch(g.exec, ctx->stream));
    ktime_end(ctx, "many", kev);
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(results, g.host_res, n_traces * sizeof(double));
    return CHAI_OK;
}
