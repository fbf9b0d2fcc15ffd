// Inline OpenCL kernels (ProgramCL): OpenCL C text -> CUDA for NVRTC, and the
// translator step that launches one.
//
// Reference: api/ProgramCL.cpp (argument kinds from the kernel signature:
// __global / image2d_t arrays, __local memory, scalars), jitast/AstOpenCL.cpp
// (the program text travels with the trace), enqueue/EnqueueOpenCL.cpp (the
// kernel is enqueued with the arrays' device buffers, the __local sizes and
// the scalars as arguments, over the NDRange the caller gave).
//
// The OpenCL C is compiled, not interpreted: a prelude maps the work-item
// functions (get_global_id ... get_num_groups), barrier / mem_fence and the
// usual type names onto CUDA; the address-space qualifiers are rewritten token
// by token (__kernel -> extern "C" __global__, __global / __private removed,
// __constant -> const, __local -> __shared__ in bodies).  A __local pointer
// parameter becomes a plain pointer that the kernel body points into its
// dynamic shared memory at the offset its size gives.
#include <cuda_runtime.h>

#include <cctype>
#include <cstring>
#include <sstream>

#include "internal.h"
#include "jit.h"
#include "trace.h"

namespace chai {

static const char* kOpenCLPrelude = R"cl(
// ---- OpenCL C on sm_100a (inline ProgramCL kernels)
typedef unsigned int uint;
typedef unsigned long long ulong;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef decltype(sizeof(0)) size_t;
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
__device__ __forceinline__ size_t get_global_id(uint d)
{ return d == 0 ? (size_t)blockIdx.x * blockDim.x + threadIdx.x
       : d == 1 ? (size_t)blockIdx.y * blockDim.y + threadIdx.y : (size_t)blockIdx.z * blockDim.z + threadIdx.z; }
__device__ __forceinline__ size_t get_local_id(uint d) { return d == 0 ? threadIdx.x : d == 1 ? threadIdx.y : threadIdx.z; }
__device__ __forceinline__ size_t get_group_id(uint d) { return d == 0 ? blockIdx.x : d == 1 ? blockIdx.y : blockIdx.z; }
__device__ __forceinline__ size_t get_local_size(uint d) { return d == 0 ? blockDim.x : d == 1 ? blockDim.y : blockDim.z; }
__device__ __forceinline__ size_t get_num_groups(uint d) { return d == 0 ? gridDim.x : d == 1 ? gridDim.y : gridDim.z; }
__device__ __forceinline__ size_t get_global_size(uint d) { return get_num_groups(d) * get_local_size(d); }
__device__ __forceinline__ uint get_work_dim() { return CHAI_CL_WORK_DIM; }
__device__ __forceinline__ void barrier(int) { __syncthreads(); }
__device__ __forceinline__ void mem_fence(int) { __threadfence_block(); }
template <class T> __device__ __forceinline__ T mad(T a, T b, T c) { return a * b + c; }
template <class T> __device__ __forceinline__ T clamp(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class T> __device__ __forceinline__ T mix(T x, T y, T a) { return x + (y - x) * a; }
#define native_exp exp
#define native_log log
#define native_sqrt sqrt
#define native_rsqrt rsqrt
#define native_sin sin
#define native_cos cos
#define native_tan tan
#define native_powr pow
#define native_exp2 exp2
#define native_log2 log2
#define half_exp exp
#define half_log log
#define half_sqrt sqrt
#define powr pow
__device__ __forceinline__ double pown(double x, int n) { return pow(x, (double)n); }
__device__ __forceinline__ float pown(float x, int n) { return powf(x, (float)n); }
__device__ __forceinline__ double rootn(double x, int n) { return pow(x, 1.0 / n); }
__device__ __forceinline__ float rootn(float x, int n) { return powf(x, 1.0f / n); }
// ---- program text
)cl";

namespace {

struct Tok {
    enum Kind { IDENT, OTHER } kind;
    std::string text;
};

// identifiers, and everything else (punctuation, numbers, white space,
// comments, literals) as opaque runs
std::vector<Tok> tokenize(const std::string& s)
{
    std::vector<Tok> out;
    size_t i = 0;
    auto other = [&](size_t a, size_t b) {
        if (!out.empty() && out.back().kind == Tok::OTHER) out.back().text.append(s, a, b - a);
        else out.push_back({Tok::OTHER, s.substr(a, b - a)});
    };
    while (i < s.size()) {
        const char c = s[i];
        if (std::isalpha((unsigned char)c) || c == '_') {
            size_t j = i + 1;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) j++;
            out.push_back({Tok::IDENT, s.substr(i, j - i)});
            i = j;
        } else if (std::isdigit((unsigned char)c)) {
            size_t j = i + 1;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '.' || s[j] == '_')) j++;
            other(i, j);
            i = j;
        } else if (c == '/' && i + 1 < s.size() && s[i + 1] == '/') {
            size_t j = s.find('\n', i);
            j = j == std::string::npos ? s.size() : j;
            other(i, j);
            i = j;
        } else if (c == '/' && i + 1 < s.size() && s[i + 1] == '*') {
            size_t j = s.find("*/", i + 2);
            j = j == std::string::npos ? s.size() : j + 2;
            other(i, j);
            i = j;
        } else if (c == '"' || c == '\'') {
            size_t j = i + 1;
            while (j < s.size() && s[j] != c) j += (s[j] == '\\') ? 2 : 1;
            j = std::min(s.size(), j + 1);
            other(i, j);
            i = j;
        } else {
            other(i, i + 1);
            i++;
        }
    }
    return out;
}

bool is_kernel_kw(const std::string& t) { return t == "__kernel" || t == "kernel"; }
bool mentions_image(const std::vector<Tok>& p)
{
    for (const Tok& x : p)
        if (x.kind == Tok::IDENT && (x.text == "image2d_t" || x.text == "image3d_t" || x.text == "sampler_t"))
            return true;
    return false;
}
bool is_local_kw(const std::string& t) { return t == "__local" || t == "local"; }

}  // namespace

// `local_bytes[i]`: bytes of the i-th argument of kernel `name` when it is a
// __local pointer (0 otherwise).
int opencl_to_cuda(const std::string& src, const std::string& name, const std::vector<size_t>& local_bytes,
                   int work_dim, std::string& out, std::string& err)
{
    std::vector<Tok> t = tokenize(src);
    std::ostringstream os;
    os << "#define CHAI_CL_WORK_DIM " << work_dim << "\n" << kOpenCLPrelude;
    bool found = false;
    for (size_t i = 0; i < t.size(); i++) {
        if (t[i].kind != Tok::IDENT) {
            os << t[i].text;
            continue;
        }
        const std::string& w = t[i].text;
        if (is_kernel_kw(w)) {
            // __kernel void NAME ( params ) {
            size_t j = i + 1;
            auto next_ident = [&](size_t& k) -> int {
                while (k < t.size() && t[k].kind == Tok::OTHER) {
                    for (char ch : t[k].text)
                        if (!std::isspace((unsigned char)ch)) return -1;
                    k++;
                }
                return k < t.size() ? (int)k : -1;
            };
            int kv = next_ident(j);
            if (kv < 0 || t[kv].text != "void") { err = "inline kernel: expected void after __kernel"; return -1; }
            j = (size_t)kv + 1;
            int kn = next_ident(j);
            if (kn < 0) { err = "inline kernel: missing kernel name"; return -1; }
            const std::string kname = t[kn].text;
            // parameters: tokens up to the matching ')'
            size_t k = (size_t)kn + 1;
            std::string pre;          // text between name and '('
            while (k < t.size() && !(t[k].kind == Tok::OTHER && t[k].text.find('(') != std::string::npos)) pre += t[k++].text;
            if (k >= t.size()) { err = "inline kernel: missing parameter list"; return -1; }
            const size_t lp = t[k].text.find('(');
            const std::string params_before = t[k].text.substr(0, lp);
            std::vector<Tok> plist;
            int depth = 1;
            std::string tail;        // text after the closing ')' within its run
            auto walk = [&](const std::string& txt) -> bool {
                std::string cur;
                for (size_t p = 0; p < txt.size(); p++) {
                    const char ch = txt[p];
                    if (ch == '(') depth++;
                    if (ch == ')' && --depth == 0) {
                        if (!cur.empty()) plist.push_back({Tok::OTHER, cur});
                        tail = txt.substr(p + 1);
                        return true;
                    }
                    cur += ch;
                }
                if (!cur.empty()) plist.push_back({Tok::OTHER, cur});
                return false;
            };
            bool closed = walk(t[k].text.substr(lp + 1));
            k++;
            while (!closed && k < t.size()) {
                if (t[k].kind == Tok::IDENT) plist.push_back(t[k]);
                else closed = walk(t[k].text);
                k++;
            }
            if (!closed) { err = "inline kernel: unbalanced parameter list"; return -1; }
            // the rest of the run holding ')' is processed next
            k--;
            t[k] = {Tok::OTHER, tail};
            // rewrite the parameters one by one (split at top-level commas)
            std::vector<std::vector<Tok>> params(1);
            for (const Tok& x : plist) {
                if (x.kind == Tok::IDENT) { params.back().push_back(x); continue; }
                std::string cur;
                for (char ch : x.text) {
                    if (ch == ',') {
                        if (!cur.empty()) params.back().push_back({Tok::OTHER, cur});
                        cur.clear();
                        params.emplace_back();
                    } else {
                        cur += ch;
                    }
                }
                if (!cur.empty()) params.back().push_back({Tok::OTHER, cur});
            }
            std::ostringstream inject;
            size_t offset = 0;
            const bool called = kname == name;
            if (called) found = true;
            std::ostringstream plist_out;
            for (size_t pi = 0; pi < params.size(); pi++) {
                bool local = false;
                std::string last_ident, type;
                std::ostringstream pout;
                for (const Tok& x : params[pi]) {
                    if (x.kind == Tok::IDENT) {
                        if (is_local_kw(x.text)) { local = true; continue; }
                        if (x.text == "__global" || x.text == "global" || x.text == "__private" ||
                            x.text == "private")
                            continue;
                        if (x.text == "__constant" || x.text == "constant") { pout << "const"; continue; }
                        if (!last_ident.empty() && last_ident != "const" && last_ident != "volatile" &&
                            last_ident != "restrict")
                            type += (type.empty() ? "" : " ") + last_ident;
                        last_ident = x.text;
                        pout << x.text;
                    } else {
                        pout << x.text;
                    }
                }
                if (mentions_image(params[pi])) {
                    err = "inline kernel: image2d_t arguments are not supported";
                    return -1;
                }
                if (local && called) {
                    const size_t bytes = pi < local_bytes.size() ? local_bytes[pi] : 0;
                    inject << " " << last_ident << " = reinterpret_cast<" << (type.empty() ? "float" : type)
                           << "*>(chai_cl_lmem + " << offset << ");";
                    offset += (bytes + 15) & ~size_t(15);
                }
                plist_out << (pi ? "," : "") << pout.str();
            }
            os << "extern \"C\" __global__ void " << kname << pre << params_before << "(" << plist_out.str() << ")";
            // body: copy up to and including the opening '{', then inject
            while (k < t.size()) {
                if (t[k].kind == Tok::OTHER) {
                    const size_t b = t[k].text.find('{');
                    if (b != std::string::npos) {
                        os << t[k].text.substr(0, b + 1);
                        if (called && offset)
                            os << " extern __shared__ __align__(16) unsigned char chai_cl_lmem[];" << inject.str();
                        t[k].text = t[k].text.substr(b + 1);
                        break;
                    }
                }
                os << t[k].text;
                k++;
            }
            i = k - 1;      // resume with the remainder of the run holding '{'
            continue;
        }
        if (w == "__global" || w == "global" || w == "__private" || w == "private") continue;
        if (w == "__constant" || w == "constant") { os << "const"; continue; }
        if (is_local_kw(w)) { os << "__shared__"; continue; }
        os << w;
    }
    if (!found) { err = "inline kernel: no __kernel named " + name; return -1; }
    out = os.str();
    return 0;
}

// Launch the inline kernel of node i: compile its program (cached by text),
// bind the arrays' storage, the scalars and the __local sizes, run it over the
// caller's NDRange.
int Translator::emit_inline(int i)
{
    const Node& nd = nodes_[i];
    const chai_inline_kernel& k = kernels_[nd.buffer];
    const bool two_d = k.global_size[1] != 0;
    for (int d = 0; d < (two_d ? 2 : 1); d++) {
        if (k.local_size[d] == 0 || k.global_size[d] % k.local_size[d] != 0)
            return fail(CHAI_ERR_INVALID, "inline kernel: local size must divide the global size");
    }
    const uint64_t lx = k.local_size[0], ly = two_d ? k.local_size[1] : 1;
    if (lx * ly > 1024) return fail(CHAI_ERR_INVALID, "inline kernel: more than 1024 work items per group");
    std::vector<size_t> lbytes(k.n_args, 0);
    size_t smem = 0;
    for (uint32_t a = 0; a < k.n_args; a++) {
        const chai_kernel_arg& g = k.args[a];
        if (g.kind == CHAI_KARG_LOCAL) {
            if (g.value < 0) return fail(CHAI_ERR_INVALID, "inline kernel: negative __local size");
            lbytes[a] = (size_t)g.value * prec_bytes(g.prec);
            smem += (lbytes[a] + 15) & ~size_t(15);
        } else if (g.kind != CHAI_KARG_ARRAY && g.kind != CHAI_KARG_SCALAR) {
            return fail(CHAI_ERR_INVALID, "inline kernel: argument kind");
        }
    }
    if (smem > 227 * 1024) return fail(CHAI_ERR_INVALID, "inline kernel: __local memory above 227 KB");
    std::string cuda, err;
    if (opencl_to_cuda(k.source, k.name, lbytes, two_d ? 2 : 1, cuda, err)) return fail(CHAI_ERR_INVALID, err);
    last_source = cuda;
    all_sources += cuda;
    void* fn = nullptr;
    int st = ctx_->jit->get(cuda, k.name, &fn);
    if (st) return st;
    if (dry_) return CHAI_OK;
    Step ks;
    ks.kind = Step::KERNEL;
    ks.fn = fn;
    ks.grid = dim3((unsigned)(k.global_size[0] / lx), (unsigned)(two_d ? k.global_size[1] / ly : 1), 1);
    ks.block = dim3((unsigned)lx, (unsigned)ly, 1);
    ks.smem = smem;
    size_t m = 0;
    for (uint32_t a = 0; a < k.n_args; a++) {
        const chai_kernel_arg& g = k.args[a];
        Step::Arg arg;
        if (g.kind == CHAI_KARG_ARRAY) {
            const Node& v = nodes_[nd.kids[m++]];
            if (!v.dev) return fail(CHAI_ERR_INVALID, "inline kernel: array argument without storage");
            arg.kind = Step::Arg::PTR;
            arg.r = ref_of(v.dev);
        } else if (g.kind == CHAI_KARG_LOCAL) {
            arg.kind = Step::Arg::PTR;      // set by the kernel body to its slice of shared memory
        } else {
            arg.kind = Step::Arg::I64;      // the argument's bytes at the start of the slot
            long long bits = 0;
            if (g.prec == CHAI_F32) {
                const float f = (float)g.value;
                memcpy(&bits, &f, 4);
            } else if (g.prec == CHAI_F64) {
                memcpy(&bits, &g.value, 8);
            } else if (g.prec == CHAI_I32) {
                const int32_t v32 = (int32_t)(int64_t)g.value;
                memcpy(&bits, &v32, 4);
            } else {
                const uint32_t v32 = (uint32_t)(int64_t)g.value;
                memcpy(&bits, &v32, 4);
            }
            arg.v = bits;
        }
        ks.args.push_back(arg);
    }
    st = exec(ks);
    if (st) return st;
    kernels_launched++;
    return CHAI_OK;
}

}  // namespace chai
