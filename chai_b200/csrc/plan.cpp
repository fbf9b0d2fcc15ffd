// Plan cache: recording and replay of a trace's device operations (plan.h).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>

#include "internal.h"
#include "jit.h"
#include "plan.h"
#include "trace.h"

namespace chai {

int launch_combine(chai_cuda_ctx* ctx, const double* partials, int nblocks, int nred, int slots,
                   void* const* outs, const int* precs, const double* scales);
int launch_transpose(chai_cuda_ctx* ctx, uint32_t prec, const void* in, void* out, int64_t w, int64_t h,
                     int64_t slots);

void plan_key(const chai_trace_desc* t, const chai_buffer_binding* b, size_t nb, std::vector<uint64_t>& key,
              std::vector<uint64_t>& ids)
{
    key.clear();
    ids.clear();
    auto ordinal = [&](uint64_t id) -> uint64_t {
        for (size_t k = 0; k < ids.size(); k++)
            if (ids[k] == id) return k;
        ids.push_back(id);
        return ids.size() - 1;
    };
    // variable numbers only name values: the key uses first-occurrence
    // ordinals, so a trace recorded again with fresh variables matches
    std::vector<uint32_t> vars;
    auto var_ordinal = [&](uint32_t v) -> uint64_t {
        for (size_t k = 0; k < vars.size(); k++)
            if (vars[k] == v) return k;
        vars.push_back(v);
        return vars.size() - 1;
    };
    key.push_back(t->num_traces);
    key.push_back(t->n_stmts);
    key.push_back(nb);
    for (size_t i = 0; i < nb; i++) {
        key.push_back(var_ordinal(b[i].variable));
        key.push_back(b[i].prec);
        key.push_back(b[i].width);
        key.push_back(b[i].height);
        key.push_back(b[i].slots);
        key.push_back(ordinal(b[i].buffer));
    }
    // inline kernels: program text, name, arguments, NDRange.  The texts go
    // into the key whole (length, then 8 bytes per word), so two programs
    // never share a plan by a hash collision.
    auto push_text = [&](const char* p) {
        const size_t n = p ? strlen(p) : 0;
        key.push_back(n);
        for (size_t i = 0; i < n; i += 8) {
            uint64_t w = 0;
            memcpy(&w, p + i, std::min<size_t>(8, n - i));
            key.push_back(w);
        }
    };
    const uint32_t nk = t->kernels ? t->n_kernels : 0;
    key.push_back(nk);
    for (uint32_t k = 0; k < nk; k++) {
        const chai_inline_kernel& kd = t->kernels[k];
        push_text(kd.source);
        push_text(kd.name);
        key.push_back(kd.n_args);
        for (uint32_t a = 0; a < kd.n_args && kd.args; a++) {
            const chai_kernel_arg& g = kd.args[a];
            uint64_t bits;
            memcpy(&bits, &g.value, 8);
            key.push_back(((uint64_t)g.kind << 32) | g.prec);
            key.push_back(g.kind == CHAI_KARG_ARRAY ? ((var_ordinal(g.variable) << 32) | g.version) : bits);
        }
        key.push_back(kd.global_size[0]);
        key.push_back(kd.global_size[1]);
        key.push_back(kd.local_size[0]);
        key.push_back(kd.local_size[1]);
    }
    for (uint32_t s = 0; s < t->n_stmts; s++) {
        const chai_stmt& st = t->stmts[s];
        key.push_back((var_ordinal(st.lhs_variable) << 32) | st.lhs_version);
        key.push_back(st.n_cells);
        for (uint32_t c = 0; c < st.n_cells; c++) {
            const chai_bc& bc = st.cells[c];
            const uint64_t code = bc.kind == CHAI_BC_VARIABLE ? var_ordinal(bc.code) : bc.code;
            key.push_back(((uint64_t)bc.kind << 56) ^ (code << 24) ^ bc.version);
            if (bc.kind == CHAI_BC_SCALAR) {
                uint64_t bits;
                memcpy(&bits, &bc.scalar, 8);
                key.push_back(bits);
            } else if (bc.kind == CHAI_BC_MEMORY) {
                key.push_back(ordinal(bc.buffer));
            }
        }
    }
}

void Translator::begin_record(const std::vector<uint64_t>& buffer_ids)
{
    recording_ = true;
    cacheable_ = true;
    buf_ids_ = buffer_ids;
    plan_.reset(new Plan());
    plan_->buf_alloc.assign(buf_ids_.size(), 0);
    plan_->buf_need.assign(buf_ids_.size(), 0);
}

std::unique_ptr<Plan> Translator::take_plan()
{
    if (!recording_ || !cacheable_ || dry_ || !plan_) return nullptr;
    plan_->temp_bytes = temp_sizes_;
    plan_->kernels = kernels_launched;
    return std::move(plan_);
}

void Translator::note_buffer(uint64_t id, size_t bytes, bool alloc)
{
    if (!recording_) return;
    for (size_t k = 0; k < buf_ids_.size(); k++) {
        if (buf_ids_[k] != id) continue;
        std::vector<size_t>& v = alloc ? plan_->buf_alloc : plan_->buf_need;
        v[k] = std::max(v[k], bytes);
        return;
    }
    cacheable_ = false;     // a buffer outside the trace's own list
}

Ref Translator::ref_of(const void* p)
{
    Ref r;
    r.raw = const_cast<void*>(p);
    if (!p) return r;
    const char* q = static_cast<const char*>(p);
    for (size_t k = 0; k < buf_ids_.size(); k++) {
        Buffer* b = find_buffer(ctx_, buf_ids_[k]);
        if (!b) continue;
        const char* base = static_cast<const char*>(b->ptr);
        if (q >= base && q < base + std::max<size_t>(b->bytes, 1)) {
            r.kind = Ref::BUFFER;
            r.idx = (uint32_t)k;
            r.off = (uint64_t)(q - base);
            return r;
        }
    }
    for (size_t k = 0; k < temps_.size(); k++) {
        const char* base = static_cast<const char*>(temps_[k]);
        if (q >= base && q < base + temp_sizes_[k]) {
            r.kind = Ref::TEMP;
            r.idx = (uint32_t)k;
            r.off = (uint64_t)(q - base);
            return r;
        }
    }
    const char* sc = static_cast<const char*>(ctx_->scratch);
    if (sc && q >= sc && q < sc + ctx_->scratch_bytes) {
        r.kind = Ref::SCRATCH;
        r.off = (uint64_t)(q - sc);
        return r;
    }
    const char* sw = reinterpret_cast<const char*>(ctx_->status_word);
    if (sw && q >= sw && q < sw + 64) {
        r.kind = Ref::STATUS;
        r.off = (uint64_t)(q - sw);
        return r;
    }
    cacheable_ = false;
    return r;
}

void* Translator::ptr_of(const Ref& r) const
{
    if (!replaying_) return r.raw;
    switch (r.kind) {
        case Ref::NONE: return nullptr;
        case Ref::BUFFER: {
            Buffer* b = find_buffer(ctx_, buf_ids_[r.idx]);
            return b ? static_cast<char*>(b->ptr) + r.off : nullptr;
        }
        case Ref::TEMP: return static_cast<char*>(temps_[r.idx]) + r.off;
        case Ref::SCRATCH: return static_cast<char*>(ctx_->scratch) + r.off;
        case Ref::STATUS: return reinterpret_cast<char*>(ctx_->status_word) + r.off;
    }
    return nullptr;
}

int Translator::exec(Step& s)
{
    int st = run_step(s);
    if (st) return st;
    if (recording_) plan_->steps.push_back(s);
    return CHAI_OK;
}

typedef CUresult (*PFN_encodeTiledP)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                      const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiledP encoder()
{
    static PFN_encodeTiledP fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiledP>(p);
    }
    return fn;
}

int Translator::run_step(const Step& s)
{
    cudaStream_t stream = ctx_->stream;
    switch (s.kind) {
        case Step::KERNEL: {
            if (s.scratch_need) {
                int st = ensure_scratch(ctx_, s.scratch_need);
                if (st) return st;
            }
            std::vector<CUtensorMap> maps(s.maps.size());
            for (size_t k = 0; k < s.maps.size(); k++) {
                memset(&maps[k], 0, sizeof(CUtensorMap));
                const TmapRec& m = s.maps[k];
                if (!m.encode) continue;
                PFN_encodeTiledP enc = encoder();
                if (!enc) return set_error(ctx_, CHAI_ERR_NO_DEVICE, "cuTensorMapEncodeTiled unavailable");
                cuuint64_t dims[3] = {m.dims[0], m.dims[1], m.dims[2]};
                cuuint64_t strides[2] = {m.strides[0], m.strides[1]};
                cuuint32_t box[3] = {m.box[0], m.box[1], m.box[2]};
                cuuint32_t estr[3] = {1, 1, 1};
                void* base = ptr_of(m.base);
                if ((reinterpret_cast<uintptr_t>(base) & 15) != 0)
                    return set_error(ctx_, CHAI_ERR_INVALID, "stencil source not 16-byte aligned");
                CUresult r = enc(&maps[k], m.dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (r != CUDA_SUCCESS) return set_error(ctx_, CHAI_ERR_INVALID, "stencil tensor map encoding failed");
            }
            std::vector<long long> vals(s.args.size());
            std::vector<void*> pvals(s.args.size());
            std::vector<void*> ptrs(s.args.size());
            for (size_t k = 0; k < s.args.size(); k++) {
                const Step::Arg& a = s.args[k];
                if (a.kind == Step::Arg::I64) {
                    vals[k] = a.v;
                    ptrs[k] = &vals[k];
                } else if (a.kind == Step::Arg::PTR) {
                    pvals[k] = ptr_of(a.r);
                    ptrs[k] = &pvals[k];
                } else {
                    ptrs[k] = &maps[a.map];
                }
            }
            cudaEvent_t kev[2];
            ktime_begin(ctx_, "trace", kev);
            int st = ctx_->jit->launch(s.fn, s.grid, s.block, s.smem, ptrs.data());
            if (st) return st;
            ktime_end(ctx_, "trace", kev);
            return CHAI_OK;
        }
        case Step::COMBINE: {
            std::vector<void*> outs(s.outs.size());
            for (size_t k = 0; k < s.outs.size(); k++) outs[k] = ptr_of(s.outs[k]);
            return launch_combine(ctx_, static_cast<const double*>(ptr_of(s.partials)), s.nblocks, s.nred, s.slots,
                                  outs.data(), s.precs.data(), s.scales.data());
        }
        case Step::GEMM: {
            chai_gemm_desc d = s.desc;
            d.a = ptr_of(s.a);
            d.b = ptr_of(s.b);
            d.c = ptr_of(s.c);
            // a trace's matmul: a small one may split K (GemmSplitK)
            ctx_->trace_gemm = true;
            const int st = launch_gemm(ctx_, &d);
            ctx_->trace_gemm = false;
            return st;
        }
        case Step::GEMV:
            return launch_gemv(ctx_, s.prec, s.trans, s.m, s.n, s.alpha, ptr_of(s.a), s.lda, ptr_of(s.b), s.beta,
                               ptr_of(s.c));
        case Step::TRANSPOSE:
            return launch_transpose(ctx_, s.prec, ptr_of(s.a), ptr_of(s.b), s.w, s.h, s.nslots);
        case Step::COPY:
            CHAI_CUDA_TRY(ctx_, cudaMemcpyAsync(ptr_of(s.a), ptr_of(s.b), s.bytes, cudaMemcpyDeviceToDevice, stream));
            return CHAI_OK;
        case Step::COPY2D:
            CHAI_CUDA_TRY(ctx_, cudaMemcpy2DAsync(ptr_of(s.a), s.dpitch, ptr_of(s.b), s.spitch, s.width, s.height,
                                                  cudaMemcpyDeviceToDevice, stream));
            return CHAI_OK;
        case Step::MEMSET:
            CHAI_CUDA_TRY(ctx_, cudaMemsetAsync(ptr_of(s.a), s.value, s.bytes, stream));
            return CHAI_OK;
    }
    return set_error(ctx_, CHAI_ERR_INVALID, "plan step");
}

int Translator::replay(const Plan& p, const std::vector<uint64_t>& buffer_ids)
{
    if (buffer_ids.size() != p.buf_alloc.size()) return 1;
    replaying_ = true;
    buf_ids_ = buffer_ids;
    for (size_t k = 0; k < buf_ids_.size(); k++) {
        if (p.buf_alloc[k]) {
            int st = alloc_buffer(ctx_, buf_ids_[k], p.buf_alloc[k]);
            if (st) return st;
        }
        if (p.buf_need[k]) {
            Buffer* b = find_buffer(ctx_, buf_ids_[k]);
            if (!b || b->bytes < p.buf_need[k]) return 1;
        }
    }
    for (size_t bytes : p.temp_bytes) {
        void* q = nullptr;
        CHAI_CUDA_TRY(ctx_, cudaMallocAsync(&q, bytes, ctx_->stream));
        temps_.push_back(q);
        temp_sizes_.push_back(bytes);
    }
    for (const Step& s : p.steps) {
        int st = run_step(s);
        if (st) return st;
    }
    kernels_launched = p.kernels;
    return CHAI_OK;
}

}  // namespace chai
