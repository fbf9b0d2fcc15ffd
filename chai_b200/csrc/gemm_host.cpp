// GEMM with its operands in host memory, streamed through the GPU.
//
// The reference multiplies arrays whose boxes live in host memory: the device
// memory manager copies A and B in, the matmul runs, C is copied back on
// read-back (memmgr/MemTransJIT.cpp:18-327, enqueue/EnqueueMatmulAuto.cpp:
// 21-404), one step after the other.  Over PCIe those copies cost more than a
// large tensor-core GEMM, so here they overlap it: B is uploaded once, A is
// uploaded in blocks of rows on a copy stream, each block's GEMM runs on the
// context stream as soon as its rows have landed, and each block of C goes
// back on a second copy stream while the next block computes.  Two device
// buffers per operand block alternate; for the tensor-core precisions B's
// operand planes are written once and shared by the block GEMMs.  Every block is an ordinary
// chai_cuda_gemm call on device buffers, and a row of C depends only on the
// same row of A, so C is bit-identical to uploading everything first.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "internal.h"
#include "tuner.h"

namespace chai {

namespace {

// per-context copy streams, events and device buffers of the streamed GEMM
struct HostGemm {
    cudaStream_t in = nullptr, out = nullptr;
    cudaEvent_t ev_b = nullptr, ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {};
    void* dev = nullptr;
    size_t bytes = 0;
};

std::map<chai_cuda_ctx*, HostGemm> g_host_gemms;     // by context
std::mutex g_host_gemms_mu;                          // guards finding / inserting / erasing an entry

HostGemm& host_gemm_of(chai_cuda_ctx* ctx)
{
    std::lock_guard<std::mutex> g(g_host_gemms_mu);
    return g_host_gemms[ctx];
}

int host_gemm_setup(chai_cuda_ctx* ctx, HostGemm& h, size_t need)
{
    if (!h.in) {
        CHAI_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&h.in, cudaStreamNonBlocking));
        CHAI_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&h.out, cudaStreamNonBlocking));
        CHAI_CUDA_TRY(ctx, cudaEventCreateWithFlags(&h.ev_b, cudaEventDisableTiming));
        for (int i = 0; i < 2; i++) {
            CHAI_CUDA_TRY(ctx, cudaEventCreateWithFlags(&h.ev_in[i], cudaEventDisableTiming));
            CHAI_CUDA_TRY(ctx, cudaEventCreateWithFlags(&h.ev_comp[i], cudaEventDisableTiming));
            CHAI_CUDA_TRY(ctx, cudaEventCreateWithFlags(&h.ev_out[i], cudaEventDisableTiming));
        }
    }
    if (h.bytes < need) {
        if (h.dev) {
            CHAI_CUDA_TRY(ctx, cudaDeviceSynchronize());
            cudaFree(h.dev);
            h.dev = nullptr;
            h.bytes = 0;
        }
        CHAI_CUDA_TRY(ctx, cudaMalloc(&h.dev, need));
        h.bytes = need;
    }
    return CHAI_OK;
}

// rows x cols elements of `es` bytes between host and device, either pitch
int copy_rows(chai_cuda_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
              size_t rows, cudaMemcpyKind kind, cudaStream_t s)
{
    if (dpitch == width && spitch == width)
        CHAI_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, width * rows, kind, s));
    else
        CHAI_CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, s));
    return CHAI_OK;
}

}  // namespace

void host_gemm_release(chai_cuda_ctx* ctx)
{
    HostGemm h;
    {
        std::lock_guard<std::mutex> g(g_host_gemms_mu);
        auto it = g_host_gemms.find(ctx);
        if (it == g_host_gemms.end()) return;
        h = it->second;
        g_host_gemms.erase(it);
    }
    if (h.in) cudaStreamSynchronize(h.in);
    if (h.out) cudaStreamSynchronize(h.out);
    if (h.dev) cudaFree(h.dev);
    for (cudaEvent_t e : {h.ev_b, h.ev_in[0], h.ev_in[1], h.ev_comp[0], h.ev_comp[1], h.ev_out[0], h.ev_out[1]})
        if (e) cudaEventDestroy(e);
    if (h.in) cudaStreamDestroy(h.in);
    if (h.out) cudaStreamDestroy(h.out);
}

}  // namespace chai

using namespace chai;

extern "C" int chai_cuda_gemm_host(chai_cuda_ctx* ctx, const chai_gemm_desc* d, int64_t block_rows)
{
    if (!ctx || !d) return CHAI_ERR_INVALID;
    if (d->trans_a || d->trans_b) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "gemm_host: transposed operands");
    if (d->batch > 1) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "gemm_host: one problem per call");
    if (d->m < 0 || d->n < 0 || d->k < 0) return set_error(ctx, CHAI_ERR_INVALID, "gemm_host: negative size");
    if (d->m == 0 || d->n == 0) return CHAI_OK;
    if (!d->a || !d->b || !d->c || d->lda < d->k || d->ldb < d->n || d->ldc < d->n)
        return set_error(ctx, CHAI_ERR_INVALID, "gemm_host: bad operand pointers or leading dimensions");
    const int prec = resolve_precision(ctx, d->precision, d->m, d->n, d->k);
    const size_t es = prec == CHAI_GEMM_FP64 ? 8 : 4;
    const long long M = d->m, N = d->n, K = d->k;
    // about eight blocks, whole 128-row tiles
    long long mb = block_rows > 0 ? block_rows : (M + 7) / 8;
    mb = std::max<long long>(128, (mb + 127) / 128 * 128);
    mb = std::min(mb, M);
    const size_t b_bytes = (size_t)K * N * es, a_blk = (size_t)mb * K * es, c_blk = (size_t)mb * N * es;
    // tensor-core precisions: B is split into its operand planes once, not per block
    const size_t p_bytes = gemm_b_planes_bytes(prec, K, N);
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    HostGemm& h = host_gemm_of(ctx);
    cudaSetDevice(ctx->device);
    int st = host_gemm_setup(ctx, h, up(b_bytes) + 2 * up(a_blk) + 2 * up(c_blk) + up(p_bytes));
    if (st) return st;
    char* base = static_cast<char*>(h.dev);
    char* db = base;
    char* da[2] = {base + up(b_bytes), base + up(b_bytes) + up(a_blk)};
    char* dc[2] = {da[1] + up(a_blk), da[1] + up(a_blk) + up(c_blk)};
    char* bplanes = p_bytes ? dc[1] + up(c_blk) : nullptr;
    const bool with_c = d->beta != 0.0;
    // the copies must not start before earlier work on the context stream
    // that may still read these buffers
    CHAI_CUDA_TRY(ctx, cudaEventRecord(h.ev_comp[0], ctx->stream));
    CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(h.in, h.ev_comp[0], 0));
    st = copy_rows(ctx, db, N * es, d->b, d->ldb * es, N * es, K, cudaMemcpyHostToDevice, h.in);
    if (st) return st;
    CHAI_CUDA_TRY(ctx, cudaEventRecord(h.ev_b, h.in));
    CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, h.ev_b, 0));
    if (bplanes) {
        st = gemm_split_b(ctx, prec, reinterpret_cast<const float*>(db), N, K, N, bplanes);
        if (st) return st;
    }
    const char* ha = static_cast<const char*>(d->a);
    char* hc = static_cast<char*>(d->c);
    long long blk = 0;
    for (long long r0 = 0; r0 < M; r0 += mb, blk++) {
        const int q = (int)(blk & 1);
        const long long rows = std::min(mb, M - r0);
        if (blk >= 2) {        // buffers q were last used by block blk - 2
            CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(h.in, h.ev_comp[q], 0));
            if (with_c) CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(h.in, h.ev_out[q], 0));
        }
        st = copy_rows(ctx, da[q], K * es, ha + (size_t)r0 * d->lda * es, d->lda * es, K * es, rows,
                       cudaMemcpyHostToDevice, h.in);
        if (!st && with_c)
            st = copy_rows(ctx, dc[q], N * es, hc + (size_t)r0 * d->ldc * es, d->ldc * es, N * es, rows,
                           cudaMemcpyHostToDevice, h.in);
        if (st) return st;
        CHAI_CUDA_TRY(ctx, cudaEventRecord(h.ev_in[q], h.in));
        CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, h.ev_in[q], 0));
        if (blk >= 2 && !with_c) CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, h.ev_out[q], 0));
        chai_gemm_desc bd = *d;
        bd.precision = prec;
        bd.m = rows;
        bd.a = da[q];
        bd.lda = K;
        bd.b = db;
        bd.ldb = N;
        bd.c = dc[q];
        bd.ldc = N;
        bd.batch = 1;
        bd.stride_a = bd.stride_b = bd.stride_c = 0;
        st = bplanes ? launch_gemm_tc_cfg(ctx, &bd, prec, nullptr, bplanes) : launch_gemm(ctx, &bd);
        if (st) return st;
        CHAI_CUDA_TRY(ctx, cudaEventRecord(h.ev_comp[q], ctx->stream));
        CHAI_CUDA_TRY(ctx, cudaStreamWaitEvent(h.out, h.ev_comp[q], 0));
        st = copy_rows(ctx, hc + (size_t)r0 * d->ldc * es, d->ldc * es, dc[q], N * es, N * es, rows,
                       cudaMemcpyDeviceToHost, h.out);
        if (st) return st;
        CHAI_CUDA_TRY(ctx, cudaEventRecord(h.ev_out[q], h.out));
    }
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(h.out));
    CHAI_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return CHAI_OK;
}
