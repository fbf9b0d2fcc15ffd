// GEMV (autotune/EvergreenMatmulMV.cpp; oracle interp/InterpMatmulBase.hpp:
// 37-47) as an HBM-bound kernel, and the transpose used by `transpose()`.
//
//   y = alpha * A x + beta * y    (A m x n row-major): one warp per row,
//       128-bit loads of A unrolled 4 deep, x through the read-only L1 path,
//       FP64 accumulation for f64 and FP32 for f32, warp-shuffle row sum.
//   y = alpha * A^T x + beta * y: each thread owns 4 (f32) / 2 (f64) adjacent
//       columns; the rows are split over blockIdx.y and the per-split column
//       partials (context scratch) are summed in split order by a second
//       kernel, so the result does not depend on scheduling.
// Algorithmic bytes per launch: m*n*sizeof(T) + (m+n)*sizeof(T) (+ y read
// when beta != 0).
#include <cuda_runtime.h>

#include "chai_trace_prelude.cuh"
#include "internal.h"
#include "tuner.h"

namespace chai {

// ------------------------------------------------- bulk-copy GEMV (A x)
// A streamed through shared memory by cp.async.bulk (the copy engine keeps
// the bytes in flight, not registers): each block owns a contiguous run of
// rows; a producer warp issues 16 KB row chunks into a 4-stage ring, 8
// consumer warps each take 16 consecutive bytes per thread of a chunk (x from
// L1), and the 256 partial sums of a row are reduced in a fixed tree.  Used
// when A, x, the row pitch and the row length are 16-byte aligned.
constexpr int GB_STAGES = 4, GB_CHUNK = 16384, GB_CONSUMERS = 8;

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(chai_k::smem_u32(dst)), "l"(src), "r"(bytes), "r"(chai_k::smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(chai_k::smem_u32(bar)) : "memory");
}

template <class T>
__global__ void __launch_bounds__((GB_CONSUMERS + 1) * 32) chai_gemv_bulk(const T* __restrict__ A, long long lda,
                                                                           const T* __restrict__ x, T* __restrict__ y,
                                                                           long long m, long long n, T alpha, T beta,
                                                                           long long rows_per_block, int* status)
{
    typedef typename std::conditional<sizeof(T) == 4, float4, double2>::type V;
    constexpr int VE = 16 / sizeof(T);                      // elements per 16 bytes
    constexpr int CE = GB_CHUNK / sizeof(T);                // elements per chunk
    constexpr int PER = CE / (GB_CONSUMERS * 32 * VE);      // 16-byte vectors per thread per chunk
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[GB_STAGES], empty[GB_STAGES];
    __shared__ T red[2][GB_CONSUMERS];
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long r0 = (long long)blockIdx.x * rows_per_block;
    const long long r1 = r0 + rows_per_block < m ? r0 + rows_per_block : m;
    const long long cpr = (n + CE - 1) / CE;                // chunks per row
    const long long jobs = r0 < r1 ? (r1 - r0) * cpr : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < GB_STAGES; s++) {
            chai_k::mbar_init(&full[s], 1);
            chai_k::mbar_init(&empty[s], GB_CONSUMERS);
        }
        abort_flag = 0;
    }
    __syncthreads();
    if (warp == GB_CONSUMERS) {
        // producer
        if (lane == 0) {
            long long issued = 0;
            for (long long j = 0; j < jobs && !abort_flag; j++) {
                const int s = (int)(j % GB_STAGES);
                const long long round = j / GB_STAGES;
                if (round > 0 && !chai_k::mbar_wait_bounded(&empty[s], (unsigned)((round - 1) & 1), status)) {
                    abort_flag = 1;
                    break;
                }
                const long long row = r0 + j / cpr, c = j % cpr;
                const long long len = (n - c * CE) < CE ? (n - c * CE) : CE;
                chai_k::mbar_expect_tx(&full[s], (unsigned)(len * sizeof(T)));
                bulk_load(smem + (size_t)s * GB_CHUNK, A + row * lda + c * CE, (unsigned)(len * sizeof(T)), &full[s]);
                issued = j + 1;
            }
            // every issued copy has landed before the block exits
            for (long long j = issued - GB_STAGES < 0 ? 0 : issued - GB_STAGES; j < issued; j++)
                chai_k::mbar_wait_bounded(&full[j % GB_STAGES], (unsigned)((j / GB_STAGES) & 1), status);
        }
        return;
    }
    // consumers
    // A wait that runs out (or another warp's) marks the warp bad: it stops
    // waiting and computing but still reaches every row's named barrier, so no
    // consumer warp can block on one that left.
    const int t = threadIdx.x;                              // 0 .. 255
    T acc = 0;
    bool bad = false;
    for (long long j = 0; j < jobs; j++) {
        const int s = (int)(j % GB_STAGES);
        if (!bad) {
            if (*reinterpret_cast<volatile int*>(&abort_flag)) bad = true;
            else if (!chai_k::mbar_wait_bounded(&full[s], (unsigned)((j / GB_STAGES) & 1), status)) {
                abort_flag = 1;
                bad = true;
            }
        }
        const long long row = r0 + j / cpr, c = j % cpr;
        if (!bad) {
            const long long len = (n - c * CE) < CE ? (n - c * CE) : CE;
            const V* av = reinterpret_cast<const V*>(smem + (size_t)s * GB_CHUNK);
            const V* xv = reinterpret_cast<const V*>(x + c * CE);
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int v = i * (GB_CONSUMERS * 32) + t;      // vector index within the chunk
                if ((long long)v * VE < len) {
                    const V a = av[v];
                    const V b = __ldg(xv + v);
                    const T* pa = reinterpret_cast<const T*>(&a);
                    const T* pb = reinterpret_cast<const T*>(&b);
#pragma unroll
                    for (int e = 0; e < VE; e++) acc = fma(pa[e], pb[e], acc);
                }
            }
        }
        // the producer's next bulk copy into this stage (async proxy) must
        // follow these generic reads of it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0 && !bad) mbar_arrive(&empty[s]);
        if (c == cpr - 1) {
            // row done: fixed-order tree over the 256 consumer threads
            T w = acc;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            const int par = (int)((row - r0) & 1);
            if (lane == 0) red[par][warp] = w;
            asm volatile("bar.sync 1, %0;" ::"n"(GB_CONSUMERS * 32));
            if (t == 0) {
                T sum = 0;
#pragma unroll
                for (int k = 0; k < GB_CONSUMERS; k++) sum += red[par][k];
                y[row] = beta == (T)0 ? alpha * sum : alpha * sum + beta * y[row];
            }
            acc = 0;
        }
    }
}

static bool gemv_bulk_ok(const void* a, long long lda, const void* x, long long n, size_t esz)
{
    return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(x)) & 15) == 0 &&
           (lda * (long long)esz) % 16 == 0 && (n * (long long)esz) % 16 == 0 && n > 0;
}

template <class T>
static int launch_gemv_bulk(chai_cuda_ctx* ctx, long long m, long long n, T alpha, const T* a, long long lda,
                            const T* x, T beta, T* y)
{
    const int smem = GB_STAGES * GB_CHUNK;
    cudaFuncSetAttribute(chai_gemv_bulk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const long long blocks = std::min<long long>(m, (long long)ctx->sm_count * 3);
    const long long rpb = (m + blocks - 1) / blocks;
    const long long grid = (m + rpb - 1) / rpb;
    chai_gemv_bulk<T><<<(unsigned)grid, (GB_CONSUMERS + 1) * 32, smem, ctx->stream>>>(a, lda, x, y, m, n, alpha,
                                                                                       beta, rpb, ctx->status_word);
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    return CHAI_OK;
}

template <class T, int WARPS, int UNROLL>
__global__ void __launch_bounds__(WARPS * 32) chai_gemv_n(const T* __restrict__ A, long long lda,
                                                          const T* __restrict__ x, T* __restrict__ y, long long m,
                                                          long long n, T alpha, T beta)
{
    typedef typename std::conditional<sizeof(T) == 4, float4, double2>::type V;
    constexpr int VE = 16 / sizeof(T);
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * WARPS + (threadIdx.x >> 5);
    if (row >= m) return;
    const T* a = A + row * lda;
    T acc = 0;
    const bool vec = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(x)) & 15) == 0;
    long long done = 0;
    if (vec) {
        const long long nv = n / VE;
        const V* av = reinterpret_cast<const V*>(a);
        const V* xv = reinterpret_cast<const V*>(x);
        long long v = lane;
        // UNROLL independent 16-byte loads of A in flight per lane
        for (; v + 32 * (UNROLL - 1) < nv; v += 32 * UNROLL) {
            V ar[UNROLL], xr[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; u++) {
                ar[u] = __ldg(av + v + 32 * u);
                xr[u] = __ldg(xv + v + 32 * u);
            }
#pragma unroll
            for (int u = 0; u < UNROLL; u++) {
                const T* pa = reinterpret_cast<const T*>(&ar[u]);
                const T* px = reinterpret_cast<const T*>(&xr[u]);
#pragma unroll
                for (int j = 0; j < VE; j++) acc = fma(pa[j], px[j], acc);
            }
        }
        for (; v < nv; v += 32) {
            V a0 = __ldg(av + v), x0 = __ldg(xv + v);
            const T* pa = reinterpret_cast<const T*>(&a0);
            const T* px = reinterpret_cast<const T*>(&x0);
#pragma unroll
            for (int j = 0; j < VE; j++) acc = fma(pa[j], px[j], acc);
        }
        done = nv * VE;
    }
    for (long long j = done + lane; j < n; j += 32) acc = fma(__ldg(a + j), __ldg(x + j), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) y[row] = beta == (T)0 ? alpha * acc : alpha * acc + beta * y[row];
}

// partial[s][j] = sum over rows of split s of x[i] * A[i][j]
template <class T>
__global__ void __launch_bounds__(256) chai_gemv_t_partial(const T* __restrict__ A, long long lda,
                                                           const T* __restrict__ x, T* __restrict__ partial,
                                                           long long m, long long n, long long rows_per_split)
{
    constexpr int VE = 16 / sizeof(T);
    const long long j0 = ((long long)blockIdx.x * 256 + threadIdx.x) * VE;
    if (j0 >= n) return;
    const long long r0 = (long long)blockIdx.y * rows_per_split;
    const long long r1 = r0 + rows_per_split < m ? r0 + rows_per_split : m;
    T acc[VE];
#pragma unroll
    for (int j = 0; j < VE; j++) acc[j] = 0;
    const bool full = j0 + VE <= n && ((lda * sizeof(T)) % 16 == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
    for (long long i = r0; i < r1; i++) {
        const T xi = __ldg(x + i);
        const T* a = A + i * lda + j0;
        if (full) {
            typedef typename std::conditional<sizeof(T) == 4, float4, double2>::type V;
            V av = __ldg(reinterpret_cast<const V*>(a));
            const T* pa = reinterpret_cast<const T*>(&av);
#pragma unroll
            for (int j = 0; j < VE; j++) acc[j] = fma(pa[j], xi, acc[j]);
        } else {
            for (int j = 0; j < VE && j0 + j < n; j++) acc[j] = fma(__ldg(a + j), xi, acc[j]);
        }
    }
    T* p = partial + (long long)blockIdx.y * n + j0;
    for (int j = 0; j < VE && j0 + j < n; j++) p[j] = acc[j];
}

template <class T>
__global__ void chai_gemv_t_finish(const T* __restrict__ partial, int splits, T* __restrict__ y, long long n,
                                   T alpha, T beta)
{
    const long long j = (long long)blockIdx.x * 256 + threadIdx.x;
    if (j >= n) return;
    T acc = 0;
    for (int s = 0; s < splits; s++) acc += partial[(long long)s * n + j];
    y[j] = beta == (T)0 ? alpha * acc : alpha * acc + beta * y[j];
}

template <class T>
static int gemv_t(chai_cuda_ctx* ctx, int trans, int64_t m, int64_t n, double alpha, const void* a, int64_t lda,
                  const void* x, double beta, void* y, const GemvCfg* cfg_in)
{
    if (!trans) {
        GemvCfg cfg;
        if (cfg_in) cfg = *cfg_in;
        else tuned_gemv_cfg(ctx, m, n, sizeof(T) == 8 ? CHAI_F64 : CHAI_F32, &cfg);
        cudaEvent_t ev[2];
        ktime_begin(ctx, "gemv", ev);
        if (cfg.warps == 0 && m > 0 && gemv_bulk_ok(a, lda, x, n, sizeof(T))) {
            const int st = launch_gemv_bulk<T>(ctx, m, n, (T)alpha, (const T*)a, lda, (const T*)x, (T)beta, (T*)y);
            if (st) return st;
            ktime_end(ctx, "gemv", ev);
            return CHAI_OK;
        }
        if (cfg.warps == 0) cfg = GemvCfg{4, 1};
#define CHAI_GV(W, U)                                                                                       \
    chai_gemv_n<T, W, U><<<(unsigned)((m + W - 1) / W), W * 32, 0, ctx->stream>>>((const T*)a, lda, (const T*)x, \
                                                                                 (T*)y, m, n, (T)alpha, (T)beta)
#define CHAI_GVU(W)                                                                                         \
    do {                                                                                                    \
        if (cfg.unroll >= 8) CHAI_GV(W, 8); else if (cfg.unroll >= 4) CHAI_GV(W, 4);                        \
        else if (cfg.unroll >= 2) CHAI_GV(W, 2); else CHAI_GV(W, 1);                                        \
    } while (0)
        if (m > 0) {
            if (cfg.warps <= 2) CHAI_GVU(2);
            else if (cfg.warps <= 4) CHAI_GVU(4);
            else if (cfg.warps <= 8) CHAI_GVU(8);
            else CHAI_GVU(16);
        }
#undef CHAI_GVU
#undef CHAI_GV
        ktime_end(ctx, "gemv", ev);
        CHAI_CUDA_TRY(ctx, cudaGetLastError());
        return CHAI_OK;
    }
    constexpr int VE = 16 / sizeof(T);
    const long long colblocks = (n + 256 * VE - 1) / (256 * VE);
    long long splits = std::max<long long>(1, (long long)ctx->sm_count * 6 / std::max<long long>(1, colblocks));
    splits = std::min<long long>(splits, std::max<long long>(1, m / 16));
    const long long rps = (m + splits - 1) / splits;
    splits = (m + rps - 1) / rps;
    if (splits < 1) splits = 1;
    int st = ensure_scratch(ctx, (size_t)splits * n * sizeof(T));
    if (st) return st;
    T* partial = static_cast<T*>(ctx->scratch);
    if (m > 0 && n > 0) {
        chai_gemv_t_partial<T><<<dim3((unsigned)colblocks, (unsigned)splits), 256, 0, ctx->stream>>>(
            (const T*)a, lda, (const T*)x, partial, m, n, rps);
        chai_gemv_t_finish<T><<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(partial, (int)splits, (T*)y, n,
                                                                                     (T)alpha, (T)beta);
    }
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    return CHAI_OK;
}

int launch_gemv_cfg(chai_cuda_ctx* ctx, uint32_t prec, int trans, int64_t m, int64_t n, double alpha, const void* a,
                    int64_t lda, const void* x, double beta, void* y, const GemvCfg* cfg)
{
    if (prec == CHAI_F32) return gemv_t<float>(ctx, trans, m, n, alpha, a, lda, x, beta, y, cfg);
    if (prec == CHAI_F64) return gemv_t<double>(ctx, trans, m, n, alpha, a, lda, x, beta, y, cfg);
    return set_error(ctx, CHAI_ERR_UNSUPPORTED, "gemv precision");
}

template <class T>
static void preload_gemv_t()
{
    cudaFuncAttributes a;
#define CHAI_GVP(W)                                                                                         \
    cudaFuncGetAttributes(&a, chai_gemv_n<T, W, 1>);                                                        \
    cudaFuncGetAttributes(&a, chai_gemv_n<T, W, 2>);                                                        \
    cudaFuncGetAttributes(&a, chai_gemv_n<T, W, 4>);                                                        \
    cudaFuncGetAttributes(&a, chai_gemv_n<T, W, 8>)
    CHAI_GVP(2);
    CHAI_GVP(4);
    CHAI_GVP(8);
    CHAI_GVP(16);
#undef CHAI_GVP
}

// Load every GEMV variant now (see preload_gemm_kernels).
void preload_gemv_kernels()
{
    preload_gemv_t<float>();
    preload_gemv_t<double>();
}

int launch_gemv(chai_cuda_ctx* ctx, uint32_t prec, int trans, int64_t m, int64_t n, double alpha, const void* a,
                int64_t lda, const void* x, double beta, void* y)
{
    return launch_gemv_cfg(ctx, prec, trans, m, n, alpha, a, lda, x, beta, y, nullptr);
}

// 32x32 tiled transpose through shared memory, per slot.
template <class T>
__global__ void chai_transpose(const T* __restrict__ in, T* __restrict__ out, long long w, long long h)
{
    __shared__ T tile[32][33];
    const long long s = blockIdx.z;
    in += s * w * h;
    out += s * w * h;
    const long long x = (long long)blockIdx.x * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const long long y = (long long)blockIdx.y * 32 + k;
        if (x < w && y < h) tile[k][threadIdx.x] = in[y * w + x];
    }
    __syncthreads();
    const long long ox = (long long)blockIdx.y * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const long long oy = (long long)blockIdx.x * 32 + k;
        if (ox < h && oy < w) out[oy * h + ox] = tile[threadIdx.x][k];
    }
}

int launch_transpose(chai_cuda_ctx* ctx, uint32_t prec, const void* in, void* out, int64_t w, int64_t h,
                     int64_t slots)
{
    dim3 grid((unsigned)((w + 31) / 32), (unsigned)((h + 31) / 32), (unsigned)slots);
    if (prec_bytes(prec) == 8) chai_transpose<double><<<grid, dim3(32, 8), 0, ctx->stream>>>((const double*)in, (double*)out, w, h);
    else chai_transpose<float><<<grid, dim3(32, 8), 0, ctx->stream>>>((const float*)in, (float*)out, w, h);
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    return CHAI_OK;
}

}  // namespace chai
