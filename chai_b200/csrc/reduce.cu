// Reductions: sum / mean / dot_product (enqueue/EnqueueReduce.cpp:21-222 runs
// one serial work item per array; interp/InterpAccum.cpp:13-70 and
// interp/InterpDotprod.cpp accumulate in double).
//
// Combine order, stated: each thread accumulates its grid-stride elements in
// FP64, a warp-shuffle tree and a shared-memory tree reduce each block to one
// partial, and chai_combine_partials adds a slot's partials in FP64 with a
// fixed block-tree order.  The grid size is a function of the array size and
// the SM count only, so a result is bit-reproducible on a given GPU model.
#include <cuda_runtime.h>

#include "internal.h"

namespace chai {

template <int NT>
__device__ __forceinline__ double block_sum_d(double x)
{
    __shared__ double sm[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
    __syncthreads();
    x = threadIdx.x < NT / 32 ? sm[threadIdx.x] : 0.0;
    if (threadIdx.x < 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    }
    return x;
}

struct CombineArgs {
    void* outs[16];
    int precs[16];
    double scales[16];
};

// grid: (slots, nred); one block sums one (reduction, slot) row of partials
__global__ void __launch_bounds__(256) chai_combine_partials(const double* __restrict__ partials, int nblocks,
                                                             int slots, CombineArgs a)
{
    const int slot = blockIdx.x, r = blockIdx.y;
    const double* p = partials + ((long long)r * slots + slot) * nblocks;
    double x = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += 256) x += p[i];
    x = block_sum_d<256>(x);
    if (threadIdx.x == 0) {
        x *= a.scales[r];
        switch (a.precs[r]) {
            case CHAI_F32: static_cast<float*>(a.outs[r])[slot] = (float)x; break;
            case CHAI_F64: static_cast<double*>(a.outs[r])[slot] = x; break;
            case CHAI_I32: static_cast<int*>(a.outs[r])[slot] = (int)(long long)x; break;
            case CHAI_U32: static_cast<unsigned*>(a.outs[r])[slot] = (unsigned)(long long)x; break;
        }
    }
}

int launch_combine(chai_cuda_ctx* ctx, const double* partials, int nblocks, int nred, int slots,
                   void* const* outs, const int* precs, const double* scales)
{
    if (nred > 16) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "more than 16 reductions in one kernel");
    CombineArgs a;
    for (int r = 0; r < nred; r++) {
        a.outs[r] = outs[r];
        a.precs[r] = precs[r];
        a.scales[r] = scales[r];
    }
    chai_combine_partials<<<dim3(slots, nred), 256, 0, ctx->stream>>>(partials, nblocks, slots, a);
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    return CHAI_OK;
}

// Per-slot partial sums of a (op 0/1) or a*b (op 2); T is the array type.
template <class T, bool DOT>
__global__ void __launch_bounds__(256) chai_reduce_partials(const T* __restrict__ a, const T* __restrict__ b,
                                                            unsigned long long n, double* __restrict__ partials)
{
    const int slot = blockIdx.y;
    const T* pa = a + (unsigned long long)slot * n;
    const T* pb = DOT ? b + (unsigned long long)slot * n : nullptr;
    double acc = 0.0;
    const unsigned long long stride = (unsigned long long)gridDim.x * 256;
    // 16-byte vector loads when the slot base is aligned
    const bool vec = ((reinterpret_cast<uintptr_t>(pa) | (DOT ? reinterpret_cast<uintptr_t>(pb) : 0)) & 15) == 0;
    constexpr int VE = 16 / sizeof(T);
    unsigned long long done = 0;
    if (vec) {
        const unsigned long long nv = n / VE;
        for (unsigned long long v = blockIdx.x * 256ull + threadIdx.x; v < nv; v += stride) {
            T x[VE], y[VE];
            *reinterpret_cast<uint4*>(x) = __ldg(reinterpret_cast<const uint4*>(pa) + v);
            if (DOT) *reinterpret_cast<uint4*>(y) = __ldg(reinterpret_cast<const uint4*>(pb) + v);
#pragma unroll
            for (int j = 0; j < VE; j++) acc += DOT ? (double)(x[j] * y[j]) : (double)x[j];
        }
        done = nv * VE;
    }
    for (unsigned long long i = done + blockIdx.x * 256ull + threadIdx.x; i < n; i += stride)
        acc += DOT ? (double)(pa[i] * pb[i]) : (double)pa[i];
    acc = block_sum_d<256>(acc);
    if (threadIdx.x == 0) partials[(unsigned long long)slot * gridDim.x + blockIdx.x] = acc;
}

int launch_reduce(chai_cuda_ctx* ctx, uint32_t op, uint32_t prec, const void* a, const void* b, uint64_t n,
                  uint32_t slots, double* dev_out)
{
    const size_t eb = prec_bytes(prec);
    if (!eb) return set_error(ctx, CHAI_ERR_INVALID, "reduce precision");
    const unsigned long long nv = (n * eb + 15) / 16;
    unsigned gx = (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>((nv + 255) / 256,
                                                         (unsigned long long)ctx->sm_count * 8 / slots + 1));
    int st = ensure_scratch(ctx, (size_t)gx * slots * sizeof(double));
    if (st) return st;
    double* partials = static_cast<double*>(ctx->scratch);
    dim3 grid(gx, slots);
    const bool dot = op == 2;
#define R(T) (dot ? chai_reduce_partials<T, true><<<grid, 256, 0, ctx->stream>>>((const T*)a, (const T*)b, n, partials) \
                  : chai_reduce_partials<T, false><<<grid, 256, 0, ctx->stream>>>((const T*)a, (const T*)b, n, partials))
    switch (prec) {
        case CHAI_F32: R(float); break;
        case CHAI_F64: R(double); break;
        case CHAI_I32: R(int); break;
        case CHAI_U32: R(unsigned); break;
    }
#undef R
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    void* outs[1] = {dev_out};
    int precs[1] = {CHAI_F64};
    double scales[1] = {op == 1 ? 1.0 / (double)n : 1.0};
    return launch_combine(ctx, partials, (int)gx, 1, (int)slots, outs, precs, scales);
}

// One block per trace: add the trace's tile partials (tiles [first, next first))
// in tile order in FP64; mean divides by n; the result is rounded to the
// reduction's precision and returned as a double.
__global__ void __launch_bounds__(256) chai_many_combine(const long long* __restrict__ tab, int stride,
                                                         const double* __restrict__ partials,
                                                         double* __restrict__ out, int mean, int prec)
{
    const int t = blockIdx.x;
    const long long ntiles = tab[0];
    const int ntr = (int)tab[1];
    const long long* row = tab + 2 + (long long)t * stride;
    const long long first = row[3];
    const long long last = t + 1 < ntr ? row[stride + 3] : ntiles;
    double x = 0.0;
    for (long long i = first + threadIdx.x; i < last; i += 256) x += partials[i];
    x = block_sum_d<256>(x);
    if (threadIdx.x == 0) {
        if (mean) x /= (double)row[0];
        if (prec == CHAI_F32) x = (double)(float)x;
        out[t] = x;
    }
}

int launch_many_combine(chai_cuda_ctx* ctx, const long long* tab, int stride, const double* partials, double* out,
                        int ntr, int mean, int prec)
{
    chai_many_combine<<<ntr, 256, 0, ctx->stream>>>(tab, stride, partials, out, mean, prec);
    return cudaGetLastError() == cudaSuccess ? CHAI_OK : CHAI_ERR_LAUNCH;
}

}  // namespace chai

// ---------------------------------------------------------------------------
// Allocation-free reduction entry point.
//
// Some callers cannot allocate device memory at the moment they need a
// reduction: code that runs while another component owns the allocator (a
// pre-sized arena, a memory pool that must not grow), or callbacks where an
// allocation could block or fail late.  chai_cuda_reduce_noalloc serves them:
// it needs no context, calls no allocator, and keeps its per-block partial
// sums in the fixed array below, which the library reserves on every GPU that
// loads it, for as long as the process runs.
//
// Limits and sharing:
//   - at most CHAI_NOALLOC_PARTIALS partial sums per call (blocks x slots);
//     a call with more slots than that is rejected;
//   - every call uses the same array, which keeps whatever the previous call
//     left in it.  Each partial is written before it is read, so nothing has
//     to start at zero -- but two calls whose kernels overlap on the GPU (on
//     different streams without ordering between them) race on the array;
//   - the first call in a CUDA context (normally the device's primary
//     context, which the runtime API uses) looks up the array's device address
//     in that context; make that first call before any stream capture begins.
//     The address is remembered per context: a caller that makes its own
//     driver-API context current gets the array's address in that context.
//   - a launch failure is reported from this call's own launches
//     (cudaLaunchKernel's return value); an error left pending by unrelated
//     earlier work is neither reported as this call's nor cleared.
#include <mutex>

#define CHAI_NOALLOC_PARTIALS 8192

static __device__ __align__(256) double chai_noalloc_partials[CHAI_NOALLOC_PARTIALS];

namespace {
typedef int (*PFN_ctxGetCurrent)(void**);   // cuCtxGetCurrent (CUresult, CUcontext*)

std::mutex g_noalloc_mu;
struct NoallocSlot {
    void* cu_ctx;
    double* ptr;
};
NoallocSlot g_noalloc_slots[64];
int g_noalloc_used = 0;
PFN_ctxGetCurrent g_ctx_get = nullptr;

void* current_cu_ctx()
{
    void* c = nullptr;
    if (g_ctx_get && g_ctx_get(&c) != 0) c = nullptr;
    return c;
}

// Device address of the partials array in the calling thread's current CUDA
// context (looked up once per context, under g_noalloc_mu).
double* noalloc_partials_ptr()
{
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_ctx_get) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return nullptr;
        g_ctx_get = reinterpret_cast<PFN_ctxGetCurrent>(fn);
    }
    void* c = current_cu_ctx();
    for (int i = 0; c && i < g_noalloc_used; i++)
        if (g_noalloc_slots[i].cu_ctx == c) return g_noalloc_slots[i].ptr;
    void* p = nullptr;
    // binds the primary context to this thread if no context is current
    if (cudaGetSymbolAddress(&p, chai_noalloc_partials) != cudaSuccess || !p) return nullptr;
    c = current_cu_ctx();
    if (c) {
        for (int i = 0; i < g_noalloc_used; i++)
            if (g_noalloc_slots[i].cu_ctx == c) return g_noalloc_slots[i].ptr;
        if (g_noalloc_used < 64) g_noalloc_slots[g_noalloc_used++] = {c, static_cast<double*>(p)};
    }
    return static_cast<double*>(p);
}

template <class T>
cudaError_t noalloc_partials_launch(bool dot, dim3 grid, cudaStream_t s, const void* a, const void* b,
                                    unsigned long long n, double* partials)
{
    const T* pa = static_cast<const T*>(a);
    const T* pb = static_cast<const T*>(b);
    void* args[] = {&pa, &pb, &n, &partials};
    const void* fn = dot ? reinterpret_cast<const void*>(&chai::chai_reduce_partials<T, true>)
                         : reinterpret_cast<const void*>(&chai::chai_reduce_partials<T, false>);
    return cudaLaunchKernel(fn, grid, dim3(256), args, 0, s);
}
}  // namespace

extern "C" int chai_cuda_reduce_noalloc(uint32_t op, uint32_t prec, const void* a, const void* b, uint64_t n,
                                        uint32_t slots, double* device_out, void* cuda_stream)
{
    using namespace chai;
    if (!a || !device_out || op > 2 || (op == 2 && !b) || slots == 0) return CHAI_ERR_INVALID;
    const size_t eb = prec_bytes(prec);
    if (!eb) return CHAI_ERR_INVALID;
    if (slots > CHAI_NOALLOC_PARTIALS) return CHAI_ERR_UNSUPPORTED;   // more partials than the fixed array holds
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CHAI_ERR_NO_DEVICE;
    double* partials = noalloc_partials_ptr();
    if (!partials) return CHAI_ERR_NO_DEVICE;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned long long nv = (n * eb + 15) / 16;
    unsigned long long gx = std::min<unsigned long long>((nv + 255) / 256, (unsigned long long)sms * 8 / slots + 1);
    // blocks x slots partials must fit the fixed array
    gx = std::min<unsigned long long>(gx, CHAI_NOALLOC_PARTIALS / slots);
    if (gx < 1) gx = 1;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    const dim3 grid((unsigned)gx, slots);
    const bool dot = op == 2;
    const unsigned long long nn = n;
    cudaError_t e = cudaSuccess;
    switch (prec) {
        case CHAI_F32: e = noalloc_partials_launch<float>(dot, grid, s, a, b, nn, partials); break;
        case CHAI_F64: e = noalloc_partials_launch<double>(dot, grid, s, a, b, nn, partials); break;
        case CHAI_I32: e = noalloc_partials_launch<int>(dot, grid, s, a, b, nn, partials); break;
        case CHAI_U32: e = noalloc_partials_launch<unsigned>(dot, grid, s, a, b, nn, partials); break;
    }
    if (e == cudaSuccess) {
        CombineArgs ca;
        ca.outs[0] = device_out;
        ca.precs[0] = CHAI_F64;
        ca.scales[0] = op == 1 ? 1.0 / (double)n : 1.0;     // n = 0: mean is 0/0 = NaN, sum and dot are 0
        const double* cp = partials;
        int nb = (int)gx, ns = (int)slots;
        void* args[] = {&cp, &nb, &ns, &ca};
        e = cudaLaunchKernel(reinterpret_cast<const void*>(&chai_combine_partials), dim3(slots, 1), dim3(256), args,
                             0, s);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();          // this call's own launch error: do not leave it pending
        return CHAI_ERR_LAUNCH;
    }
    return CHAI_OK;
}
