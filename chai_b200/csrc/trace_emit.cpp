// Code emission for trace kernel groups, linear-algebra lowering and
// read-backs (second half of the trace translator, see trace.cpp).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <set>
#include <sstream>

#include "internal.h"
#include "jit.h"
#include "trace.h"
#include "tuner.h"

namespace chai {

int launch_combine(chai_cuda_ctx* ctx, const double* partials, int nblocks, int nred, int slots,
                   void* const* outs, const int* precs, const double* scales);
int launch_transpose(chai_cuda_ctx* ctx, uint32_t prec, const void* in, void* out, int64_t w, int64_t h,
                     int64_t slots);

static const char* ctype_of(int prec)
{
    switch (prec) {
        case CHAI_U32: return "unsigned";
        case CHAI_I32: return "int";
        case CHAI_F32: return "float";
        case CHAI_F64: return "double";
    }
    return "float";
}

// Exact literal of `v` in precision `prec`.
static std::string literal(double v, int prec)
{
    char buf[64];
    switch (prec) {
        case CHAI_U32: snprintf(buf, sizeof buf, "%uu", (unsigned)(uint32_t)(int64_t)v); break;
        case CHAI_I32: snprintf(buf, sizeof buf, "(int)%d", (int)(int64_t)v); break;
        case CHAI_F32: {
            float f = (float)v;
            uint32_t u;
            memcpy(&u, &f, 4);
            snprintf(buf, sizeof buf, "__int_as_float(0x%08xu)", u);
            break;
        }
        default: {
            uint64_t u;
            memcpy(&u, &v, 8);
            snprintf(buf, sizeof buf, "__longlong_as_double(0x%016" PRIx64 "ull)", u);
            break;
        }
    }
    return buf;
}

struct KArg {
    enum { PTR, I64, REF } kind;
    void* ptr;        // PTR: the device pointer passed; REF: address of the by-value argument
    long long v;
};

typedef CUresult (*PFN_encodeTiledT)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                      const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiledT tensor_map_encoder()
{
    static PFN_encodeTiledT fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiledT>(p);
    }
    return fn;
}

// stencil tile geometry (outputs per CTA: TX x TY; halo: PX columns, R rows)
constexpr int ST_TX = 128, ST_PX = 4;

int Translator::emit_group(const std::vector<int>& roots)
{
    // stencil tile height (rows of outputs per CTA; a multiple of 8): the
    // StencilRows setting, or (0, the default) chosen below per kernel
    int ST_TY = ctx_->cfg.stencil_rows > 0 ? std::max(8, std::min(64, ctx_->cfg.stencil_rows / 8 * 8)) : 32;
    const Node& r0 = nodes_[roots[0]];
    uint64_t W = r0.W, H = r0.H;
    uint32_t S = r0.slots;
    if (r0.kind == Node::REDUCE) {
        W = 1; H = 1;
        for (int k : r0.kids) { W = std::max(W, nodes_[k].W); H = std::max(H, nodes_[k].H); }
    }
    const long long n = (long long)(W * H);
    if (n == 0) return CHAI_OK;
    bool vec = (n % 4) == 0;
    std::set<int> root_set(roots.begin(), roots.end());

    // body nodes in dependency order; loads for values computed elsewhere
    std::vector<int> body;
    std::set<int> loads, seen;
    struct Sten { int src, cx, cy; };
    std::map<int, Sten> sten;
    std::function<void(int)> dfs = [&](int i) {
        if (seen.count(i)) return;
        seen.insert(i);
        const Node& nd = nodes_[i];
        const bool external = (materialize_[i] && !root_set.count(i)) || nd.kind == Node::INPUT ||
                              nd.kind == Node::MAKE;
        if (external) {
            loads.insert(i);
            body.push_back(i);
            return;
        }
        if (nd.kind == Node::GATHER) {
            // a stencil gather reads its staged window: its index expressions
            // are not evaluated
            if (!sten.count(i))
                for (size_t k = 1; k < nd.kids.size(); k++) dfs(nd.kids[k]);
        } else {
            for (int k : nd.kids) dfs(k);
        }
        body.push_back(i);
    };
    for (int r : roots) dfs(r);

    // Constant-offset stencil gathers -- the reference's "eligible gather"
    // (jitast/AstGather.cpp:90-195), which it reads through image2d_t:
    // gather{1,2}_floor(A, X + cx [, Y + cy]) where X, Y are the iteration's own
    // index arrays (f32, f64 or i32) and A has the iteration's shape.  When every
    // gather of the group is one, the group runs as 2-D tiles of TX x TY outputs
    // whose source tile plus halo is staged in shared memory: by one TMA load for
    // interior tiles, by wrapped (periodic) loads for border tiles.
    std::vector<int> srcs;
    int R = 0;
    bool mode2d = W >= 16 && H >= 4 && W < (1u << 24) && H < (1u << 24) && S <= 65535;
    bool any_gather = false;
    std::function<bool(int, int, long long&)> offset_of = [&](int x, int dim, long long& off) -> bool {
        const Node& nx = nodes_[x];
        if (nx.prec != CHAI_F32 && nx.prec != CHAI_F64 && nx.prec != CHAI_I32) return false;
        if (nx.kind == Node::CONVERT) return offset_of(nx.kids[0], dim, off);
        if (nx.kind == Node::INDEX) {
            off = 0;
            return nx.dim == dim && nx.W == W && nx.H == H;
        }
        if (nx.kind == Node::OP && (nx.op == 11 || nx.op == 14) && nx.kids.size() == 2) {
            auto ilit = [&](int k, long long& c) {
                const Node& sn = nodes_[k];
                if (sn.kind != Node::SCALAR || sn.scalar != std::floor(sn.scalar) || std::fabs(sn.scalar) > 4) return false;
                c = (long long)sn.scalar;
                return true;
            };
            long long c, o;
            if (ilit(nx.kids[1], c) && offset_of(nx.kids[0], dim, o)) {
                off = nx.op == 11 ? o + c : o - c;
                return true;
            }
            if (nx.op == 11 && ilit(nx.kids[0], c) && offset_of(nx.kids[1], dim, o)) {
                off = o + c;
                return true;
            }
        }
        return false;
    };
    size_t tile_bytes = 0;
    for (int i : body) {
        const Node& nd = nodes_[i];
        if (nd.kind != Node::GATHER) continue;
        any_gather = true;
        const Node& a = nodes_[nd.kids[0]];
        long long cx = 0, cy = 0;
        bool ok = a.W == W && a.H == H && offset_of(nd.kids[1], 0, cx) &&
                  (nd.op == 40 || offset_of(nd.kids[2], 1, cy)) && std::llabs(cx) <= ST_PX && std::llabs(cy) <= 4;
        if (!ok) { mode2d = false; break; }
        sten[i] = Sten{nd.kids[0], (int)cx, (int)cy};
        if (std::find(srcs.begin(), srcs.end(), nd.kids[0]) == srcs.end()) srcs.push_back(nd.kids[0]);
        R = std::max(R, (int)std::llabs(cy));
    }
    auto tile_bytes_for = [&](int ty) {
        size_t b = 0;
        for (int src : srcs) b += (size_t)(ty + 2 * R) * (ST_TX + 2 * ST_PX) * prec_bytes(nodes_[src].prec);
        return b;
    };
    // Default height: 64 rows when the staged tiles fit the 46 KiB of static
    // shared memory and the image still gives every SM four tiles, else 32.
    // Taller tiles stage fewer halo rows per output (Kirsch 8192^2: 126.2 us
    // at 64 rows, 126.8 at 48, 132.4 at 32, 158.4 at 16).
    if (ctx_->cfg.stencil_rows <= 0) {
        const long long tiles64 = (long long)((W + ST_TX - 1) / ST_TX) * (long long)((H + 63) / 64) * S;
        ST_TY = (tile_bytes_for(64) <= 46 * 1024 && tiles64 >= 4LL * ctx_->sm_count) ? 64 : 32;
    }
    tile_bytes = tile_bytes_for(ST_TY);
    mode2d = mode2d && any_gather && srcs.size() <= 2 && tile_bytes <= 46 * 1024;
    if (!mode2d) sten.clear();
    if (mode2d) {
        body.clear();
        loads.clear();
        seen.clear();
        for (int r : roots) dfs(r);
    }
    const int SH = ST_TY + 2 * R, SW = ST_TX + 2 * ST_PX;
    // Output rows per stencil thread (StencilRowsPerThread; each thread: RY
    // rows x 4 columns).  The rows of a thread share their staged windows --
    // the row at offset d serves the gathers at cy = d - q of every row q.
    // Default 1: on the Kirsch trace two rows issue as many instructions per
    // output as one (63.8 against 63.3) at 58 instead of 40 registers, and
    // run 3 % slower.  Groups with generators or reductions keep one row
    // (their per-element order is tied to 4-element vectors).
    int RY = 1;
    if (mode2d) {
        bool simple = true;
        for (int i : body)
            if (nodes_[i].kind == Node::RNG || nodes_[i].kind == Node::REDUCE) simple = false;
        const int want = std::max(1, std::min(4, ctx_->cfg.stencil_rows_per_thread));
        if (simple)
            for (int ry = want; ry > 1; ry /= 2)
                if (ST_TY % (8 * ry) == 0) { RY = ry; break; }
    }
    const int NV = 4 * RY;   // values per thread and node
    const std::string JL = "for (int j = 0; j < " + std::to_string(NV) + "; j++)";
    std::map<std::pair<int, int>, int> win_lo, win_hi;   // (source tile, row offset) -> column range
    std::set<std::pair<int, int>> win_done;
    for (auto& kv : sten) {
        const int k = (int)(std::find(srcs.begin(), srcs.end(), kv.second.src) - srcs.begin());
        for (int q = 0; q < RY; q++) {
            const std::pair<int, int> wk(k, kv.second.cy + q);
            if (!win_lo.count(wk)) { win_lo[wk] = kv.second.cx; win_hi[wk] = kv.second.cx; }
            win_lo[wk] = std::min(win_lo[wk], kv.second.cx);
            win_hi[wk] = std::max(win_hi[wk], kv.second.cx);
        }
    }
    const bool use_tma = mode2d && (W % 4) == 0;
    std::vector<TmapRec> tmaps;

    // Max of monotone affine maps.  A tree of chai max ops (`a < b ? b : a`)
    // whose leaves are all c * s_k - t, with one constant c >= 1 and one node
    // t, equals c * m - t where m is the same tree over the s_k, bit for bit,
    // whenever t is not infinite: s -> fl(fl(c s) - t) is monotone
    // non-decreasing (rounding is monotone, c > 0), NaNs sit at the same
    // leaves in both trees, two leaves with equal values have equal bits
    // (with c >= 1, c s rounds to zero only for s = +-0, so the only
    // signed-zero result, -0, comes from s = -0 and t = +0 and ties no larger
    // s), and a NaN t makes every leaf the canonical NaN.  The kernel takes
    // the short form per element and the original tree when t is infinite
    // (inf - inf would break monotonicity).  Saves, per output of an n-leaf
    // tree, n - 1 multiplies and n - 1 subtractions (Kirsch: 14 of ~63).
    // f32 trees go one step further: with t finite and non-zero and no NaN
    // among the s_k, the chai tree's pick equals the IEEE maximum in value,
    // and a zero of either sign gives c * (+-0) - t = -t, so the tree runs as
    // max.NaN.f32 (one instruction per node instead of compare + select),
    // whose NaN result sends the element to the original tree.
    struct MaxAffine {
        int t = -1, c = -1;
        bool c_first = true;
        std::string fast, slow, nanfast;   // the tree over s_k / over c * s_k - t / over s_k by max.NaN, element j
    };
    std::map<int, MaxAffine> fused;
    std::set<int> absorbed;
    if (ctx_->cfg.fuse_max_affine) {
        std::map<int, int> uses;
        for (int i : body)
            for (int k : nodes_[i].kids) uses[k]++;
        for (int r : roots) uses[r]++;
        for (auto it = body.rbegin(); it != body.rend(); ++it) {
            const int r = *it;
            const Node& rn = nodes_[r];
            if (absorbed.count(r) || loads.count(r) || rn.kind != Node::OP || rn.op != 302 || rn.kids.size() != 2 ||
                (rn.prec != CHAI_F32 && rn.prec != CHAI_F64))
                continue;
            const int P = rn.prec;
            const char* TT = ctype_of(P);
            MaxAffine m;
            std::vector<int> inner;
            auto own = [&](int k) { return uses[k] == 1 && !root_set.count(k) && !loads.count(k); };
            std::function<bool(int, bool, std::string&, std::string&, std::string&)> walk =
                [&](int k, bool top, std::string& fs, std::string& ss, std::string& ns) -> bool {
                const Node& n = nodes_[k];
                if (n.kind == Node::OP && n.op == 302 && n.kids.size() == 2 && n.prec == P && (top || own(k))) {
                    std::string f0, s0, n0, f1, s1, n1;
                    if (!walk(n.kids[0], false, f0, s0, n0) || !walk(n.kids[1], false, f1, s1, n1)) return false;
                    if (!top) inner.push_back(k);
                    fs = std::string("f2<302, ") + TT + ">(" + f0 + ", " + f1 + ")";
                    ss = std::string("f2<302, ") + TT + ">(" + s0 + ", " + s1 + ")";
                    ns = "max_nan(" + n0 + ", " + n1 + ")";
                    return true;
                }
                // leaf: sub(mul(c, s), t) (or mul(s, c)), owned by the tree
                if (top || !own(k) || n.kind != Node::OP || n.op != 14 || n.kids.size() != 2 || n.prec != P) return false;
                const int mk = n.kids[0], tk = n.kids[1];
                const Node& mn = nodes_[mk];
                if (!own(mk) || mn.kind != Node::OP || mn.op != 13 || mn.kids.size() != 2 || mn.prec != P ||
                    nodes_[tk].prec != P)
                    return false;
                int ck = -1, sk = -1;
                bool c_first = true;
                for (int side = 0; side < 2; side++) {
                    const Node& cn = nodes_[mn.kids[side]];
                    if (cn.kind != Node::SCALAR) continue;
                    const double cv = P == CHAI_F32 ? (double)(float)cn.scalar : cn.scalar;
                    if (!(cv >= 1.0) || std::isinf(cv)) continue;
                    ck = mn.kids[side];
                    sk = mn.kids[1 - side];
                    c_first = side == 0;
                    break;
                }
                if (ck < 0 || nodes_[sk].prec != P) return false;
                if (m.t < 0) {
                    m.t = tk;
                    m.c = ck;
                    m.c_first = c_first;
                } else if (m.t != tk || nodes_[m.c].scalar != nodes_[ck].scalar) {
                    return false;
                }
                inner.push_back(k);
                inner.push_back(mk);
                const std::string vs = "v" + std::to_string(sk) + "[j]", vc = "v" + std::to_string(ck) + "[j]";
                fs = vs;
                ns = vs;
                ss = std::string("f2<14, ") + TT + ">(f2<13, " + TT + ">(" + (c_first ? vc + ", " + vs : vs + ", " + vc) +
                     "), v" + std::to_string(tk) + "[j])";
                return true;
            };
            std::string fs, ss, ns;
            if (!walk(r, true, fs, ss, ns) || m.t < 0) continue;
            m.fast = fs;
            m.slow = ss;
            if (P == CHAI_F32) m.nanfast = ns;
            fused[r] = m;
            for (int k : inner) absorbed.insert(k);
        }
    }
    std::ostringstream os;
    std::vector<KArg> args;
    args.push_back({KArg::I64, nullptr, n});
    args.push_back({KArg::I64, nullptr, (long long)W});
    args.push_back({KArg::I64, nullptr, (long long)H});
    os << "extern \"C\" __global__ void __launch_bounds__(256";
    // stencil kernels: StencilMinBlocks CTAs per SM if set; a fused max tree
    // keeps its sums live across the finiteness test, so those kernels ask
    // for 5 (48 registers: 54 otherwise, 4 CTAs per SM, 4 % slower on Kirsch)
    const int min_blocks = ctx_->cfg.stencil_min_blocks > 0 ? ctx_->cfg.stencil_min_blocks : fused.empty() ? 0 : 5;
    if (mode2d && min_blocks > 0) os << ", " << min_blocks;
    os << ") chai_group(const long long n, const long long W, const long long H";
    bool need_xy = false;
    for (int i : body) {
        const Node& nd = nodes_[i];
        if (loads.count(i)) {
            os << ", const " << ctype_of(nd.prec) << "* __restrict__ p" << i;
            args.push_back({KArg::PTR, nd.dev, 0});
            if (!(nd.W == W && nd.H == H) && !(nd.W == 1 && nd.H == 1)) need_xy = true;
        }
        if (nd.kind == Node::INDEX || nd.kind == Node::GATHER) need_xy = true;
        if (nd.kind == Node::RNG) {
            const uint64_t vl = nd.prec == CHAI_F64 ? 2 : 4;
            if (!vec || (nd.W % vl) != 0) need_xy = true;
        }
        if (nd.kind == Node::GATHER) {
            const Node& a = nodes_[nd.kids[0]];
            os << ", const " << ctype_of(a.prec) << "* __restrict__ g" << i;
            args.push_back({KArg::PTR, a.dev, 0});
        }
    }
    int nred = 0;
    std::vector<int> reds;
    for (int r : roots) {
        const Node& nd = nodes_[r];
        if (nd.kind == Node::REDUCE) {
            reds.push_back(r);
            nred++;
        } else {
            os << ", " << ctype_of(nd.prec) << "* __restrict__ o" << r;
            args.push_back({KArg::PTR, nd.dev, 0});
        }
    }
    os << ", double* __restrict__ partials";
    if (mode2d) {
        os << ", int* __restrict__ status";
        for (size_t k = 0; k < srcs.size(); k++) os << ", const __grid_constant__ chai_k::Tmap tm" << k;
    }
    os << ")\n{\n";
    os << "  using namespace chai_ops; using namespace chai_rng;\n";
    // Per-thread accumulators: FP64 (the interpreter's accumulator type,
    // interp/InterpAccum.cpp) by default; ReduceAccum=f32 keeps the
    // per-thread partial sums of f32 reductions in f32 (block tree and the
    // combine stay FP64) -- an option that trades accuracy for issue slots,
    // measured against the default on the Monte Carlo trace
    std::vector<bool> red_f32(reds.size(), false);
    for (size_t k = 0; k < reds.size(); k++) {
        const Node& nd = nodes_[reds[k]];
        bool f = ctx_->cfg.reduce_accum_f32;
        for (int kid : nd.kids) f = f && nodes_[kid].prec == CHAI_F32;
        red_f32[k] = f;
    }
    if (nred) os << "  double red[" << nred << "] = {0};\n";
    if (std::find(red_f32.begin(), red_f32.end(), true) != red_f32.end())
        os << "  float redf[" << nred << "] = {0};\n";
    if (!mode2d) {
        os << "  const int slot = blockIdx.y;\n";
        os << "  const long long nchunk = (n + 3) >> 2;\n";
        os << "  for (long long c = (long long)blockIdx.x * 256 + threadIdx.x; c < nchunk; "
              "c += (long long)gridDim.x * 256) {\n";
        os << "    const long long e0 = c << 2;\n";
        if (!vec) os << "    bool ok[4]; for (int j = 0; j < 4; j++) ok[j] = e0 + j < n;\n";
        if (need_xy)
            os << "    long long xx[4], yy[4]; { const long long y0 = e0 / W, x0 = e0 - y0 * W; "
                  "for (int j = 0; j < 4; j++) { long long x = x0 + j, y = y0; while (x >= W) { x -= W; y++; } "
                  "xx[j] = x; yy[j] = y; } }\n";
    } else {
        vec = (W % 4) == 0;
        os << "  const int slot = blockIdx.z;\n";
        os << "  const long long tx0 = (long long)blockIdx.x * " << ST_TX << ", ty0 = (long long)blockIdx.y * " << ST_TY
           << ";\n";
        for (size_t k = 0; k < srcs.size(); k++)
            os << "  __shared__ __align__(128) " << ctype_of(nodes_[srcs[k]].prec) << " tile" << k << "[" << SH * SW
               << "];\n";
        os << "  __shared__ __align__(8) unsigned long long tbar;\n";
        os << "  bool tile_ok = true;\n";
        os << "  {\n    const bool interior = " << (use_tma ? "true" : "false") << " && tx0 - " << ST_PX
           << " >= 0 && tx0 + " << ST_TX + ST_PX << " <= W && ty0 - " << R << " >= 0 && ty0 + " << ST_TY + R
           << " <= H;\n";
        // Border tiles: with StencilBorderTma (an image at least one tile
        // large) they are staged by the same TMA load, whose rows and columns
        // outside the image arrive zero-filled, and only those elements are
        // then replaced by wrapped loads; otherwise every element of a border
        // tile is a wrapped load.
        const bool border_tma = use_tma && ctx_->cfg.stencil_border_tma && W >= (uint64_t)SW && H >= (uint64_t)SH;
        os << "    if (" << (border_tma ? "true" : "interior")
           << ") {\n      if (threadIdx.x == 0) chai_k::mbar_init(&tbar, 1);\n      __syncthreads();\n"
              "      if (threadIdx.x == 0) {\n        chai_k::mbar_expect_tx(&tbar, " << tile_bytes << "u);\n";
        for (size_t k = 0; k < srcs.size(); k++) {
            const Node& a = nodes_[srcs[k]];
            os << "        chai_k::tma_load_3d(tile" << k << ", &tm" << k << ", &tbar, (int)(tx0 - " << ST_PX
               << "), (int)(ty0 - " << R << "), slot % " << a.slots << ");\n";
        }
        os << "      }\n      tile_ok = chai_k::mbar_wait_bounded(&tbar, 0, status);\n";
        os << (border_tma ? "    }\n    if (!interior && tile_ok) {\n" : "    } else {\n");
        for (size_t k = 0; k < srcs.size(); k++) {
            const Node& a = nodes_[srcs[k]];
            const long long sl = a.slots > 1 ? (long long)(a.W * a.H) : 0;
            int gsrc = -1;   // the pointer parameter of a gather reading this source
            for (auto& kv : sten)
                if (kv.second.src == srcs[k]) { gsrc = kv.first; break; }
            os << "      for (int idx = threadIdx.x; idx < " << SH * SW << "; idx += 256) { const int r = idx / " << SW
               << ", c = idx - r * " << SW << "; ";
            if (border_tma)
                os << "const long long y = ty0 - " << R << " + r, x = tx0 - " << ST_PX
                   << " + c; if (y >= 0 && y < H && x >= 0 && x < W) continue; ";
            os << "tile" << k << "[idx] = g" << gsrc << "[(long long)(slot % "
               << a.slots << ") * " << sl << " + chai_k::wrapn(ty0 - " << R << " + r, H) * W + chai_k::wrapn(tx0 - "
               << ST_PX << " + c, W)]; }\n";
        }
        os << "    }\n    __syncthreads();\n  }\n";
        os << "  const int lx = (threadIdx.x & 31) * 4;\n";
        os << "  for (int rr = 0; rr < " << ST_TY / (8 * RY) << " && tile_ok; rr++) {\n";
        os << "    const int ly = " << RY << " * ((threadIdx.x >> 5) + 8 * rr);\n";
        os << "    const long long yv = ty0 + ly, xv = tx0 + lx;\n";
        os << "    if (yv >= H || xv >= W) continue;\n";
        os << "    const long long e0 = yv * W + xv;\n";
        os << "    bool ok[" << NV << "]; long long xx[" << NV << "], yy[" << NV << "];\n";
        os << "    " << JL << " { ok[j] = xv + (j & 3) < W && yv + (j >> 2) < H; xx[j] = xv + (j & 3); "
              "yy[j] = yv + (j >> 2); }\n";
    }
    const double two_pi = 2.0 * ctx_->cfg.rng_pi;
    const int layout = ctx_->cfg.rng_layout;
    for (int i : body) {
        const Node& nd = nodes_[i];
        const char* T = ctype_of(nd.prec);
        if (absorbed.count(i)) continue;
        os << "    " << T << " v" << i << "[" << NV << "];\n";
        if (fused.count(i)) {
            // the test per element (one per thread for all its elements
            // issued fewer instructions, 53.9 against 56.1 per Kirsch output,
            // but left less independent work: 155.4 against 148.6 us)
            const MaxAffine& m = fused[i];
            const std::string vc = "v" + std::to_string(m.c) + "[j]";
            const std::string cm = m.c_first ? vc + ", m" : "m, " + vc;
            if (!m.nanfast.empty())
                os << "    " << JL << " { const " << T << " m = " << m.nanfast << "; const " << T << " t = v" << m.t
                   << "[j]; if (!isinf(t) && t != (" << T << ")0 && !isnan(m)) v" << i << "[j] = f2<14, " << T
                   << ">(f2<13, " << T << ">(" << cm << "), t); else v" << i << "[j] = " << m.slow << "; }\n";
            else
                os << "    " << JL << " { if (!isinf(v" << m.t << "[j])) { const " << T << " m = " << m.fast << "; v" << i
                   << "[j] = f2<14, " << T << ">(f2<13, " << T << ">(" << cm << "), v" << m.t << "[j]); } else v" << i
                   << "[j] = " << m.slow << "; }\n";
            continue;
        }
        if (loads.count(i)) {
            const long long sl = nd.slots > 1 ? (long long)(nd.W * nd.H) : 0;
            std::string sbase = "(long long)(slot % " + std::to_string(nd.slots) + ") * " + std::to_string(sl);
            if (nd.W == W && nd.H == H) {
                if (vec && RY == 1) os << "    chai_k::ld4(p" << i << " + " << sbase << " + e0, v" << i << ");\n";
                else if (vec)
                    for (int q = 0; q < RY; q++)
                        os << "    if (yv + " << q << " < H) chai_k::ld4p(p" << i << " + " << sbase << " + e0 + " << q
                           << " * W, v" << i << " + " << 4 * q << "); else for (int j = 0; j < 4; j++) v" << i
                           << "[" << 4 * q << " + j] = (" << T << ")0;\n";
                else
                    os << "    " << JL << " v" << i << "[j] = ok[j] ? p" << i << "[" << sbase
                       << " + e0 + (j >> 2) * W + (j & 3)] : (" << T << ")0;\n";
            } else if (nd.W == 1 && nd.H == 1) {
                os << "    { const " << T << " t = p" << i << "[slot % " << nd.slots
                   << "]; " << JL << " v" << i << "[j] = t; }\n";
            } else {
                os << "    " << JL << " v" << i << "[j] = p" << i << "[" << sbase << " + (yy[j] % "
                   << nd.H << ") * " << nd.W << " + (xx[j] % " << nd.W << ")];\n";
            }
            continue;
        }
        switch (nd.kind) {
            case Node::SCALAR:
            case Node::FILL: {
                const std::string lit = literal(nd.scalar, nd.prec);
                os << "    " << JL << " v" << i << "[j] = " << lit << ";\n";
                break;
            }
            case Node::CONVERT:
                os << "    " << JL << " v" << i << "[j] = (" << T << ")v" << nd.kids[0] << "[j];\n";
                break;
            case Node::INDEX:
                os << "    " << JL << " v" << i << "[j] = (" << T << ")("
                   << (nd.dim == 0 ? "xx" : "yy") << "[j] % " << (nd.dim == 0 ? nd.W : nd.H) << ");\n";
                break;
            case Node::OP: {
                const int ar = (int)nd.kids.size();
                if (nd.op == 23) {
                    os << "    " << JL << " v" << i << "[j] = (v" << nd.kids[0] << "[j] != 0) ? ("
                       << T << ")v" << nd.kids[1] << "[j] : (" << T << ")v" << nd.kids[2] << "[j];\n";
                    break;
                }
                // f32 add / sub as packed f32x2 pairs.  Multiplies stay scalar: ptxas
                // fuses a packed mul.rn.f32x2 feeding a packed add / sub into a packed
                // FMA (one rounding instead of two), which would change results;
                // scalar mul.rn.f32 results feeding packed add / sub are not fused.
                // In a stencil the operands of a gather whose column offset is odd
                // relative to its window straddle register pairs and are re-paired
                // by moves (PackF32Stencil).
                if (ctx_->cfg.pack_f32 && (!mode2d || ctx_->cfg.pack_f32_stencil) && ar == 2 &&
                    nd.prec == CHAI_F32 && (nd.op == 11 || nd.op == 14) && nodes_[nd.kids[0]].prec == CHAI_F32 &&
                    nodes_[nd.kids[1]].prec == CHAI_F32) {
                    for (int q = 0; q < NV / 4; q++)
                        os << "    f2x4<" << nd.op << ">(v" << nd.kids[0] << " + " << 4 * q << ", v" << nd.kids[1]
                           << " + " << 4 * q << ", v" << i << " + " << 4 * q << ");\n";
                    break;
                }
                // operand precision: widest operand (fp-only ops at least f32);
                // predicates return 1/0 in that precision
                os << "    " << JL << " v" << i << "[j] = f" << ar << "<" << nd.op << ", " << T
                   << ">(";
                for (int k = 0; k < ar; k++)
                    os << (k ? ", " : "") << "(" << T << ")v" << nd.kids[k] << "[j]";
                os << ");\n";
                break;
            }
            case Node::GATHER: {
                if (sten.count(i)) {
                    // all gathers of one (source, absolute row offset) share one
                    // window of the staged row: columns lx + PX + cmin .. lx + PX +
                    // 3 + cmax, read with 16-byte shared loads where aligned (lx and
                    // the tile pitch are multiples of 4 elements); row q of the
                    // thread reads the window at row offset cy + q
                    const Sten& g = sten[i];
                    const int k = (int)(std::find(srcs.begin(), srcs.end(), g.src) - srcs.begin());
                    const char* ST = ctype_of(nodes_[g.src].prec);
                    const int ve = 16 / (int)prec_bytes(nodes_[g.src].prec);
                    for (int q = 0; q < RY; q++) {
                        const std::pair<int, int> wkey(k, g.cy + q);
                        const int cmin = win_lo[wkey], cmax = win_hi[wkey];
                        const int b0 = ST_PX + cmin, w = 4 + cmax - cmin;
                        const std::string wn = "w" + std::to_string(k) + "_" + std::to_string(g.cy + q + 8);
                        if (!win_done.count(wkey)) {
                            win_done.insert(wkey);
                            os << "    " << ST << " " << wn << "[" << w << "]; { const " << ST << "* rowp = tile" << k
                               << " + (ly + " << R + g.cy + q << ") * " << SW << " + lx;\n";
                            for (int t = 0; t < w;) {
                                if ((b0 + t) % ve == 0 && t + ve <= w) {
                                    os << "      chai_k::lds_vec(rowp + " << b0 + t << ", " << wn << " + " << t << ");\n";
                                    t += ve;
                                } else {
                                    os << "      " << wn << "[" << t << "] = rowp[" << b0 + t << "];\n";
                                    t++;
                                }
                            }
                            os << "    }\n";
                        }
                        os << "    for (int j = 0; j < 4; j++) v" << i << "[" << 4 * q << " + j] = " << wn << "[j + "
                           << g.cx - cmin << "];\n";
                    }
                    break;
                }
                const Node& a = nodes_[nd.kids[0]];
                const long long sl = a.slots > 1 ? (long long)(a.W * a.H) : 0;
                os << "    for (int j = 0; j < 4; j++) { const long long base = (long long)(slot % " << a.slots
                   << ") * " << sl << "; ";
                if (nd.op == 40)
                    os << "const long long gx = gather_index(v" << nd.kids[1] << "[j], " << a.W
                       << "); const long long gy = yy[j] % " << a.H << "; ";
                else
                    os << "const long long gx = gather_index(v" << nd.kids[1] << "[j], " << a.W
                       << "); const long long gy = gather_index(v" << nd.kids[2] << "[j], " << a.H << "); ";
                if (!vec) os << "if (!ok[j]) { v" << i << "[j] = 0; continue; } ";
                os << "v" << i << "[j] = g" << i << "[base + gy * " << a.W << " + gx]; }\n";
                break;
            }
            case Node::RNG: {
                const bool f64 = nd.prec == CHAI_F64;
                const uint64_t vl = f64 ? 2 : 4;
                const uint64_t vw = (nd.W + vl - 1) / vl;   // vectors per (padded) row
                const std::string tmpl = "<" + std::to_string(nd.variant) + ", " + std::to_string(layout) + ">";
                const std::string slotbase = "(unsigned long long)(slot % " + std::to_string(nd.slots) + ") * " +
                                             std::to_string(vw * nd.H);
                const unsigned long long seed = f64 ? nd.seed : (uint32_t)nd.seed;
                std::ostringstream conv;   // lane value from raw lane(s)
                if (!f64) {
                    // 32-bit generators
                    auto lane_expr = [&](const std::string& raw, const std::string& lane) {
                        std::ostringstream e;
                        if (nd.prec == CHAI_U32) e << "(unsigned)(" << raw << ")." << lane;
                        else if (nd.prec == CHAI_I32) e << "(int)(" << raw << ")." << lane;
                        else e << "u01_f32((" << raw << ")." << lane << ")";
                        return e.str();
                    };
                    if (vec && nd.W % 4 == 0) {
                        os << "    { const u32x4 r = raw32" << tmpl << "((unsigned)(" << slotbase << " + (e0 >> 2)), "
                           << seed << "u, true);\n";
                        if (nd.dist == 1) {
                            os << "      box_muller_f32(u01_f32(r.x), u01_f32(r.y), " << literal(two_pi, CHAI_F32)
                               << ", v" << i << "[0], v" << i << "[1]);\n";
                            os << "      box_muller_f32(u01_f32(r.z), u01_f32(r.w), " << literal(two_pi, CHAI_F32)
                               << ", v" << i << "[2], v" << i << "[3]);\n";
                        } else {
                            os << "      v" << i << "[0] = " << lane_expr("r", "x") << "; v" << i << "[1] = "
                               << lane_expr("r", "y") << "; v" << i << "[2] = " << lane_expr("r", "z") << "; v" << i
                               << "[3] = " << lane_expr("r", "w") << ";\n";
                        }
                        os << "    }\n";
                    } else {
                        // generic: one generator call per element, pick its lane
                        os << "    for (int j = 0; j < 4; j++) { const unsigned long long tid = " << slotbase
                           << " + (unsigned long long)yy[j] * " << vw << " + (unsigned long long)xx[j] / 4; "
                           << "const int ln = (int)(xx[j] & 3); const u32x4 r = raw32" << tmpl
                           << "((unsigned)tid, " << seed << "u, true); const unsigned a[4] = {r.x, r.y, r.z, r.w}; ";
                        if (nd.dist == 1)
                            os << "float z0, z1; box_muller_f32(u01_f32(a[ln & 2]), u01_f32(a[(ln & 2) + 1]), "
                               << literal(two_pi, CHAI_F32) << ", z0, z1); v" << i << "[j] = (ln & 1) ? z1 : z0; }\n";
                        else if (nd.prec == CHAI_F32)
                            os << "v" << i << "[j] = u01_f32(a[ln]); }\n";
                        else
                            os << "v" << i << "[j] = (" << T << ")a[ln]; }\n";
                    }
                } else {
                    if (vec && nd.W % 2 == 0) {
                        os << "    for (int h = 0; h < 2; h++) { const u64x2 r = raw64" << tmpl << "(" << slotbase
                           << " + (unsigned long long)(e0 >> 1) + h, " << seed << "ull);\n";
                        if (nd.dist == 1)
                            os << "      box_muller_f64(u01_f64(r.x), u01_f64(r.y), " << literal(two_pi, CHAI_F64)
                               << ", v" << i << "[2 * h], v" << i << "[2 * h + 1]); }\n";
                        else
                            os << "      v" << i << "[2 * h] = u01_f64(r.x); v" << i << "[2 * h + 1] = u01_f64(r.y); }\n";
                    } else {
                        os << "    for (int j = 0; j < 4; j++) { const unsigned long long tid = " << slotbase
                           << " + (unsigned long long)yy[j] * " << vw << " + (unsigned long long)xx[j] / 2; "
                           << "const int ln = (int)(xx[j] & 1); const u64x2 r = raw64" << tmpl << "(tid, " << seed
                           << "ull); ";
                        if (nd.dist == 1)
                            os << "double z0, z1; box_muller_f64(u01_f64(r.x), u01_f64(r.y), " << literal(two_pi, CHAI_F64)
                               << ", z0, z1); v" << i << "[j] = ln ? z1 : z0; }\n";
                        else
                            os << "v" << i << "[j] = u01_f64(ln ? r.y : r.x); }\n";
                    }
                }
                if (nd.limits && nd.dist == 0 && (nd.prec == CHAI_F32 || nd.prec == CHAI_F64)) {
                    // EnqueueAST.cpp:532-543: u * (max - min) [+ min]
                    const double len = nd.hi - nd.lo;
                    if (nd.prec == CHAI_F32) {
                        os << "    for (int j = 0; j < 4; j++) { float t = __fmul_rn(v" << i << "[j], "
                           << literal(len, CHAI_F32) << ");";
                        if (nd.lo != 0.0) os << " t = __fadd_rn(t, " << literal(nd.lo, CHAI_F32) << ");";
                        os << " v" << i << "[j] = t; }\n";
                    } else {
                        os << "    for (int j = 0; j < 4; j++) { double t = __dmul_rn(v" << i << "[j], "
                           << literal(len, CHAI_F64) << ");";
                        if (nd.lo != 0.0) os << " t = __dadd_rn(t, " << literal(nd.lo, CHAI_F64) << ");";
                        os << " v" << i << "[j] = t; }\n";
                    }
                }
                break;
            }
            case Node::REDUCE:
                break;   // accumulated below
            default:
                return fail(CHAI_ERR_UNSUPPORTED, "node kind in element kernel");
        }
    }
    // reductions
    for (int k = 0; k < nred; k++) {
        const Node& nd = nodes_[reds[k]];
        const Node& a = nodes_[nd.kids[0]];
        std::string term;
        if (red_f32[k]) {
            term = nd.op == 130 ? "v" + std::to_string(nd.kids[0]) + "[j] * v" + std::to_string(nd.kids[1]) + "[j]"
                                : "v" + std::to_string(nd.kids[0]) + "[j]";
            os << "    for (int j = 0; j < 4; j++) " << (vec ? "" : "if (ok[j]) ") << "redf[" << k << "] += " << term
               << ";\n";
            continue;
        }
        if (nd.op == 130) {
            const Node& b = nodes_[nd.kids[1]];
            (void)b;
            // each product in the operands' common type, summed in FP64, as
            // the interpreter accumulates (interp/InterpDotprod.cpp:40-138)
            term = "chai_k::dot_term(v" + std::to_string(nd.kids[0]) + "[j], v" + std::to_string(nd.kids[1]) + "[j])";
        } else {
            (void)a;
            term = "(double)v" + std::to_string(nd.kids[0]) + "[j]";
        }
        os << "    for (int j = 0; j < 4; j++) " << (vec ? "" : "if (ok[j]) ") << "red[" << k << "] += " << term
           << ";\n";
    }
    // stores
    for (int r : roots) {
        const Node& nd = nodes_[r];
        if (nd.kind == Node::REDUCE) continue;
        if (vec && RY == 1) os << "    chai_k::st4(o" << r << " + (long long)slot * n + e0, v" << r << ");\n";
        else if (vec)
            for (int q = 0; q < RY; q++)
                os << "    if (yv + " << q << " < H) chai_k::st4p(o" << r << " + (long long)slot * n + e0 + " << q
                   << " * W, v" << r << " + " << 4 * q << ");\n";
        else
            os << "    " << JL << " if (ok[j]) o" << r << "[(long long)slot * n + e0 + (j >> 2) * W + (j & 3)] = v" << r
               << "[j];\n";
    }
    os << "  }\n";
    if (nred) {
        for (int k = 0; k < nred; k++)
            if (red_f32[k]) os << "  red[" << k << "] = (double)redf[" << k << "];\n";
        os << "  chai_k::block_sum<" << nred << ", 256>(red);\n";
        if (!mode2d)
            os << "  if (threadIdx.x == 0) for (int k = 0; k < " << nred << "; k++) partials[((long long)k * gridDim.y + "
                  "slot) * gridDim.x + blockIdx.x] = red[k];\n";
        else
            os << "  if (threadIdx.x == 0) for (int k = 0; k < " << nred << "; k++) partials[((long long)k * gridDim.z + "
                  "slot) * (gridDim.x * gridDim.y) + blockIdx.y * gridDim.x + blockIdx.x] = red[k];\n";
    }
    os << "}\n";

    last_source = os.str();
    all_sources += last_source;
    void* fn = nullptr;
    int st = ctx_->jit->get(last_source, "chai_group", &fn);
    if (st) return st;
    if (dry_) return CHAI_OK;
    const long long nchunk = (n + 3) / 4;
    long long gx = (nchunk + 255) / 256, gy = 1;
    const long long cap = std::max<long long>(1, (long long)ctx_->sm_count * 8 / (long long)S);
    gx = std::min(gx, cap);
    if (mode2d) {
        gx = ((long long)W + ST_TX - 1) / ST_TX;
        gy = ((long long)H + ST_TY - 1) / ST_TY;
        if (gy > 65535) return fail(CHAI_ERR_UNSUPPORTED, "stencil grid too tall");
    }
    const long long nblocks = gx * gy;
    double* partials = nullptr;
    if (nred) {
        st = ensure_scratch(ctx_, (size_t)nred * S * nblocks * sizeof(double));
        if (st) return st;
        partials = static_cast<double*>(ctx_->scratch);
    }
    const size_t n_checked = args.size();
    args.push_back({KArg::PTR, partials, 0});
    if (mode2d) {
        args.push_back({KArg::PTR, ctx_->status_word, 0});
        for (size_t k = 0; k < srcs.size(); k++) {
            TmapRec m;
            if (use_tma) {
                const Node& a = nodes_[srcs[k]];
                const size_t eb = prec_bytes(a.prec);
                m.encode = true;
                m.dt = a.prec == CHAI_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                       : a.prec == CHAI_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                       : a.prec == CHAI_I32 ? CU_TENSOR_MAP_DATA_TYPE_INT32
                                            : CU_TENSOR_MAP_DATA_TYPE_UINT32;
                m.dims[0] = a.W; m.dims[1] = a.H; m.dims[2] = a.slots;
                m.strides[0] = a.W * eb; m.strides[1] = a.W * a.H * eb;
                m.box[0] = (uint32_t)SW; m.box[1] = (uint32_t)SH; m.box[2] = 1;
                m.base = ref_of(a.dev);
            }
            tmaps.push_back(m);
            args.push_back({KArg::REF, nullptr, 0});
        }
    }
    for (size_t k = 0; k < n_checked; k++)
        if (args[k].kind == KArg::PTR && !args[k].ptr)
            return fail(CHAI_ERR_INVALID, "trace kernel operand without storage");
    Step ks;
    ks.kind = Step::KERNEL;
    ks.fn = fn;
    ks.grid = mode2d ? dim3((unsigned)gx, (unsigned)gy, S) : dim3((unsigned)gx, S, 1);
    ks.block = dim3(256, 1, 1);
    ks.scratch_need = nred ? (size_t)nred * S * nblocks * sizeof(double) : 0;
    for (size_t k = 0; k < args.size(); k++) {
        Step::Arg a;
        if (args[k].kind == KArg::I64) {
            a.kind = Step::Arg::I64;
            a.v = args[k].v;
        } else if (args[k].kind == KArg::PTR) {
            a.kind = Step::Arg::PTR;
            a.r = ref_of(args[k].ptr);
        } else {
            a.kind = Step::Arg::TMAP;
            a.map = (int)ks.maps.size();
            ks.maps.push_back(tmaps[ks.maps.size()]);
        }
        ks.args.push_back(a);
    }
    st = exec(ks);
    if (st) return st;
    kernels_launched++;
    if (nred) {
        Step cs;
        cs.kind = Step::COMBINE;
        cs.partials = ref_of(partials);
        cs.nblocks = (int)nblocks;
        cs.nred = nred;
        cs.slots = (int)S;
        for (int r : reds) {
            const Node& nd = nodes_[r];
            cs.outs.push_back(ref_of(nd.dev));
            cs.precs.push_back(nd.prec);
            cs.scales.push_back(nd.op == 131 ? 1.0 / (double)n : 1.0);
        }
        st = exec(cs);
        if (st) return st;
        kernels_launched++;
    }
    return CHAI_OK;
}

int Translator::emit_linalg(int i)
{
    Node& nd = nodes_[i];
    if (dry_) return CHAI_OK;
    if (nd.kind == Node::TRANSPOSE) {
        const Node& a = nodes_[nd.kids[0]];
        kernels_launched++;
        Step ts;
        ts.kind = Step::TRANSPOSE;
        ts.prec = a.prec;
        ts.a = ref_of(a.dev);
        ts.b = ref_of(nd.dev);
        ts.w = (int64_t)a.W;
        ts.h = (int64_t)a.H;
        ts.nslots = a.slots;
        return exec(ts);
    }
    const Node& l = nodes_[nd.kids[0]];
    const Node& r = nodes_[nd.kids[1]];
    if (l.prec != r.prec || (l.prec != CHAI_F32 && l.prec != CHAI_F64))
        return fail(CHAI_ERR_UNSUPPORTED, "matmul needs two f32 or two f64 operands");
    const int prec = l.prec;
    const size_t eb = prec_bytes(prec);
    const int gp = prec == CHAI_F64 ? CHAI_GEMM_FP64 : CHAI_GEMM_AUTO;
    const int64_t batch = std::max(l.slots, r.slots);
    const int64_t sl = l.slots > 1 ? (int64_t)(l.W * l.H) : 0, sr = r.slots > 1 ? (int64_t)(r.W * r.H) : 0;
    const int64_t so = (int64_t)(nd.W * nd.H);
    double beta = 0.0, alpha = 1.0;
    if (nd.kind == Node::MATMULG) {
        const Node& c = nodes_[nd.kids[2]];
        if (c.prec != prec) return fail(CHAI_ERR_UNSUPPORTED, "matmul C precision");
        Step cp;
        cp.kind = Step::COPY;
        cp.a = ref_of(nd.dev);
        cp.b = ref_of(c.dev);
        cp.bytes = node_bytes(nd);
        int st = exec(cp);
        if (st) return st;
        alpha = nd.alpha;
        beta = nd.beta;
    }
    kernels_launched++;
    if (l.H > 1 && r.H > 1) {
        if (l.W != r.H) return fail(CHAI_ERR_INVALID, "matmul inner dimensions differ");
        chai_gemm_desc d{};
        d.precision = gp;
        d.m = (int64_t)l.H; d.n = (int64_t)r.W; d.k = (int64_t)l.W;
        d.a = l.dev; d.lda = (int64_t)l.W;
        d.b = r.dev; d.ldb = (int64_t)r.W;
        d.c = nd.dev; d.ldc = (int64_t)nd.W;
        d.alpha = alpha; d.beta = beta;
        d.batch = batch; d.stride_a = sl; d.stride_b = sr; d.stride_c = so;
        Step gs;
        gs.kind = Step::GEMM;
        gs.desc = d;
        gs.a = ref_of(d.a);
        gs.b = ref_of(d.b);
        gs.c = ref_of(d.c);
        return exec(gs);
    }
    // matrix-vector / vector-matrix / outer product: per slot
    for (int64_t s = 0; s < batch; s++) {
        const char* A = static_cast<const char*>(l.dev) + (size_t)(s * sl) * eb;
        const char* B = static_cast<const char*>(r.dev) + (size_t)(s * sr) * eb;
        char* C = static_cast<char*>(nd.dev) + (size_t)(s * so) * eb;
        int st;
        if (l.H == 1 && r.H == 1) {
            chai_gemm_desc d{};
            d.precision = prec == CHAI_F64 ? CHAI_GEMM_FP64 : CHAI_GEMM_FP32;
            d.m = (int64_t)l.W; d.n = (int64_t)r.W; d.k = 1;
            d.a = A; d.lda = 1; d.b = B; d.ldb = (int64_t)r.W; d.c = C; d.ldc = (int64_t)r.W;
            d.alpha = alpha; d.beta = beta; d.batch = 1;
            Step gs;
            gs.kind = Step::GEMM;
            gs.desc = d;
            gs.a = ref_of(d.a);
            gs.b = ref_of(d.b);
            gs.c = ref_of(d.c);
            st = exec(gs);
        } else {
            Step vs;
            vs.kind = Step::GEMV;
            vs.prec = prec;
            vs.alpha = alpha;
            vs.beta = beta;
            vs.c = ref_of(C);
            if (r.H == 1) {
                if (l.W != r.W) return fail(CHAI_ERR_INVALID, "matvec length differs");
                vs.trans = 0; vs.m = (int64_t)l.H; vs.n = (int64_t)l.W; vs.lda = (int64_t)l.W;
                vs.a = ref_of(A); vs.b = ref_of(B);
            } else {
                if (l.W != r.H) return fail(CHAI_ERR_INVALID, "vecmat length differs");
                vs.trans = 1; vs.m = (int64_t)r.H; vs.n = (int64_t)r.W; vs.lda = (int64_t)r.W;
                vs.a = ref_of(B); vs.b = ref_of(A);
            }
            st = exec(vs);
        }
        if (st) return st;
    }
    return CHAI_OK;
}

int Translator::do_read(int i)
{
    const Node& rd = nodes_[i];
    const Node& v = nodes_[rd.kids[0]];
    const size_t eb = prec_bytes(v.prec);
    const size_t vl = v.prec == CHAI_F64 ? 2 : 4;
    size_t need = rd.read_kind == 0 ? vl * eb * v.slots : node_bytes(v);
    int st = alloc_buffer(ctx_, rd.buffer, need);
    if (st) return st;
    note_buffer(rd.buffer, need, true);
    Buffer* dst = find_buffer(ctx_, rd.buffer);
    if (rd.read_kind == 0) {
        // read_scalar: the reference's FrontMem holds vecLength partials that
        // the client adds (api/ArrayFP.cpp:86-104); here the first is the
        // full value and the rest are zero.
        Step ms;
        ms.kind = Step::MEMSET;
        ms.a = ref_of(dst->ptr);
        ms.bytes = need;
        st = exec(ms);
        if (st) return st;
        Step cs;
        cs.kind = Step::COPY2D;
        cs.a = ref_of(dst->ptr);
        cs.dpitch = vl * eb;
        cs.b = ref_of(v.dev);
        cs.spitch = (size_t)(v.W * v.H) * eb;
        cs.width = eb;
        cs.height = v.slots;
        return exec(cs);
    }
    Step cs;
    cs.kind = Step::COPY;
    cs.a = ref_of(dst->ptr);
    cs.b = ref_of(v.dev);
    cs.bytes = need;
    return exec(cs);
}

}  // namespace chai

using namespace chai;

// Replay of a recorded plan from a captured CUDA graph (the reference keys
// repeated work by trace hash, runtime/Scheduler.cpp:48-89, and re-runs its
// statement pipeline each time).  The plan's buffers are allocated first; the
// graph is captured once for a set of device pointers (the trace's buffers,
// the context scratch and status word) and launched whenever the same
// pointers come back -- one launch for the whole trace, temporaries allocated
// and freed inside the graph.  Returns 0 when the graph ran, > 0 when the
// plain replay should run instead (the plan does not fit, or the capture was
// not possible), < 0 on error.
static int graph_replay(chai_cuda_ctx* ctx, uint64_t h, const Plan& p, const std::vector<uint64_t>& ids)
{
    if (ids.size() != p.buf_alloc.size()) return 1;
    std::vector<void*> sig;
    for (size_t k = 0; k < ids.size(); k++) {
        if (p.buf_alloc[k]) {
            int st = alloc_buffer(ctx, ids[k], p.buf_alloc[k]);
            if (st) return st;
        }
        Buffer* b = find_buffer(ctx, ids[k]);
        if (p.buf_need[k] && (!b || b->bytes < p.buf_need[k])) return 1;
        sig.push_back(b ? b->ptr : nullptr);
    }
    sig.push_back(ctx->scratch);
    sig.push_back(ctx->status_word);
    sig.push_back(ctx->stream);
    chai_cuda_ctx::PlanGraph& g = ctx->graphs[h];
    if (!g.exec || g.sig != sig) {
        // capture on the second consecutive replay with these pointers: a
        // trace whose buffers change every evaluation (fresh uploads) keeps
        // the plain replay instead of paying a capture per call
        if (g.pending != sig) {
            g.pending = sig;
            return 1;
        }
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.sig.clear();
        cudaGraph_t graph = nullptr;
        std::lock_guard<std::mutex> cap(ctx->capture_mutex);
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return 1;
        }
        ctx->capturing = true;
        int st;
        {
            Translator tr(ctx);
            st = tr.replay(p, ids);
        }   // temporaries freed inside the capture
        ctx->capturing = false;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (st != 0 || e != cudaSuccess || !graph) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return 1;                                  // run the plain replay instead
        }
        e = cudaGraphInstantiateWithFlags(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            g.exec = nullptr;
            cudaGetLastError();
            return 1;
        }
        g.sig = sig;
    }
    CHAI_CUDA_TRY(ctx, cudaGraphLaunch(g.exec, ctx->stream));
    ctx->graph_launches++;
    return 0;
}

extern "C" int chai_cuda_evaluate(chai_cuda_ctx* ctx, const chai_trace_desc* t, const chai_buffer_binding* b,
                                  size_t nb)
{
    if (!ctx || !t || (!t->stmts && t->n_stmts) || (!b && nb)) return CHAI_ERR_INVALID;
    if (fault_injected("evaluate")) return set_error(ctx, CHAI_ERR_INJECTED, "injected evaluate failure");
    cudaSetDevice(ctx->device);
    std::vector<uint64_t> key, ids;
    uint64_t h = 0;
    if (ctx->cfg.plan_cache) {
        plan_key(t, b, nb, key, ids);
        h = 1469598103934665603ull;                       // FNV-1a over the key words
        for (uint64_t w : key) { h ^= w; h *= 1099511628211ull; }
        auto it = ctx->plans.find(h);
        if (it != ctx->plans.end() && it->second->key == key) {
            const bool graphs = ctx->cfg.plan_graph == 1 || (ctx->cfg.plan_graph < 0 && !ctx->kernel_timing);
            if (graphs) {
                int gst = graph_replay(ctx, h, *it->second, ids);
                if (gst < 0) return gst;
                if (gst == 0) {
                    ctx->plan_hits++;
                    return CHAI_OK;
                }
            }
            Translator tr(ctx);
            int st = tr.replay(*it->second, ids);
            if (st < 0) return st;
            if (st == 0) {
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) return cuda_status(ctx, e, "evaluate");
                ctx->plan_hits++;
                return CHAI_OK;
            }
        }
    }
    Translator tr(ctx);
    if (ctx->cfg.plan_cache) tr.begin_record(ids);
    int st = tr.run(t, b, nb);
    if (st) return st;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(ctx, e, "evaluate");
    if (ctx->cfg.plan_cache) {
        std::unique_ptr<Plan> p = tr.take_plan();
        if (p) {
            if (ctx->plans.size() >= 1024) {
                ctx->plans.clear();
                for (auto& kv : ctx->graphs)
                    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
                ctx->graphs.clear();
            }
            auto g = ctx->graphs.find(h);          // a graph of an earlier plan with this hash
            if (g != ctx->graphs.end()) {
                if (g->second.exec) cudaGraphExecDestroy(g->second.exec);
                ctx->graphs.erase(g);
            }
            p->key = std::move(key);
            ctx->plans[h] = std::shared_ptr<Plan>(std::move(p));
        }
    }
    return CHAI_OK;
}

// Diagnostic counterpart of the reference's logged kernel source
// (kernel/KernelCache.cpp:82-89 prints the generated OpenCL when built with
// --log): plans the trace, emits every element kernel and compiles each with
// NVRTC for sm_100a.  Needs no device; allocates and launches nothing.
extern "C" int chai_cuda_trace_source(const chai_trace_desc* t, const chai_buffer_binding* b, size_t nb,
                                      const char* config, char* out, size_t cap, size_t* needed)
{
    if (!t || (!t->stmts && t->n_stmts) || (!b && nb)) return CHAI_ERR_INVALID;
    static thread_local std::string last_err;
    chai_cuda_ctx ctx;
    ctx.device = -1;
    parse_config(ctx.cfg, config);
    ctx.jit.reset(new Jit(&ctx));
    ctx.jit->set_compile_only(true);
    Translator tr(&ctx, true);
    int st = tr.run(t, b, nb);
    const std::string& src = st ? ctx.last_error : tr.all_sources;
    if (needed) *needed = src.size() + 1;
    if (out && cap) {
        const size_t k = std::min(cap - 1, src.size());
        memcpy(out, src.data(), k);
        out[k] = 0;
    }
    return st;
}

extern "C" int chai_cuda_trace_shapes(const chai_trace_desc* t, const chai_buffer_binding* b, size_t nb,
                                      chai_value_shape* out, size_t cap, size_t* count)
{
    if (!t || (!t->stmts && t->n_stmts) || (!b && nb) || (!out && cap)) return CHAI_ERR_INVALID;
    chai_cuda_ctx ctx;
    ctx.device = -1;
    Translator tr(&ctx, true);
    int st = tr.parse_all(t, b, nb);
    if (st) return st;
    const std::vector<chai_value_shape>& v = tr.statement_values();
    if (count) *count = v.size();
    for (size_t i = 0; i < v.size() && i < cap; i++) out[i] = v[i];
    return CHAI_OK;
}
