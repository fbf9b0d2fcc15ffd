// CUDA-core GEMM: the FP32 FFMA baseline (and FP64 DFMA for Arrayd64
// traces).  C = alpha * A B + beta * C, row-major, strided batch.  This is the
// "plain FP32" arm of the GEMM precision sweep that the tensor-core paths
// (gemm_tc.cu) are measured against; the reference's counterpart is the
// auto-tuned Evergreen kernel (autotune/EvergreenMatmulMM.cpp), whose
// register blocking (blockH x blockW per work item, optional local-memory
// tiles) this kernel fixes at 8x8 per thread over a 128x128x8 block tile.
#include <cuda_runtime.h>

#include "internal.h"

namespace chai {

template <class T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
chai_gemm_simt(const T* __restrict__ A, const T* __restrict__ B, T* __restrict__ C, long long M, long long N,
               long long K, long long lda, long long ldb, long long ldc, T alpha, T beta, long long sa,
               long long sb, long long sc)
{
    constexpr int NT = (BM / TM) * (BN / TN);
    __shared__ T As[2][BK][BM];
    __shared__ T Bs[2][BK][BN];
    const long long z = blockIdx.z;
    A += z * sa;
    B += z * sb;
    C += z * sc;
    const long long m0 = (long long)blockIdx.y * BM, n0 = (long long)blockIdx.x * BN;
    const int tid = threadIdx.x;
    const int tr = tid / (BN / TN), tc = tid % (BN / TN);
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = 0;
    // loaders: A tile BM x BK, B tile BK x BN
    constexpr int A_PER = BM * BK / NT, B_PER = BK * BN / NT;
    T ra[A_PER], rb[B_PER];
    auto load = [&](long long k0) {
#pragma unroll
        for (int e = 0; e < A_PER; e++) {
            const int idx = tid + e * NT;
            const int r = idx / BK, c = idx % BK;
            const long long gm = m0 + r, gk = k0 + c;
            ra[e] = (gm < M && gk < K) ? A[gm * lda + gk] : (T)0;
        }
#pragma unroll
        for (int e = 0; e < B_PER; e++) {
            const int idx = tid + e * NT;
            const int r = idx / BN, c = idx % BN;
            const long long gk = k0 + r, gn = n0 + c;
            rb[e] = (gk < K && gn < N) ? B[gk * ldb + gn] : (T)0;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int e = 0; e < A_PER; e++) {
            const int idx = tid + e * NT;
            As[buf][idx % BK][idx / BK] = ra[e];
        }
#pragma unroll
        for (int e = 0; e < B_PER; e++) {
            const int idx = tid + e * NT;
            Bs[buf][idx / BN][idx % BN] = rb[e];
        }
    };
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (long long k0 = 0; k0 < K; k0 += BK) {
        const bool more = k0 + BK < K;
        if (more) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) a[i] = As[buf][kk][tr * TM + i];
#pragma unroll
            for (int j = 0; j < TN; j++) b[j] = Bs[buf][kk][tc * TN + j];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (more) {
            store(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const long long gm = m0 + tr * TM + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const long long gn = n0 + tc * TN + j;
            if (gn >= N) continue;
            T* c = C + gm * ldc + gn;
            *c = beta == (T)0 ? alpha * acc[i][j] : alpha * acc[i][j] + beta * *c;
        }
    }
}

int launch_gemm_simt(chai_cuda_ctx* ctx, const chai_gemm_desc* d)
{
    const long long batch = d->batch > 0 ? d->batch : 1;
    if (d->trans_a || d->trans_b) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "simt gemm: transposed operands");
    if (d->m == 0 || d->n == 0) return CHAI_OK;
    if (d->precision == CHAI_GEMM_FP64) {
        dim3 grid((unsigned)((d->n + 63) / 64), (unsigned)((d->m + 63) / 64), (unsigned)batch);
        chai_gemm_simt<double, 64, 64, 8, 4, 4><<<grid, 256, 0, ctx->stream>>>(
            (const double*)d->a, (const double*)d->b, (double*)d->c, d->m, d->n, d->k, d->lda, d->ldb, d->ldc,
            d->alpha, d->beta, d->stride_a, d->stride_b, d->stride_c);
    } else {
        // Small products (C1's 512 x 512 gives 16 tiles of 128 x 128) leave most
        // SMs idle: take 64 x 64, then 32 x 64 tiles until the grid covers the
        // SMs; their K step is 32 wide, so a short K loop waits on fewer
        // rounds of global loads.  Every variant runs each output's FMA chain in the same k order,
        // so the results are bit-identical whichever tile is chosen.
        auto tiles = [&](long long bm, long long bn) { return ((d->m + bm - 1) / bm) * ((d->n + bn - 1) / bn) * batch; };
#define CHAI_SIMT(BMV, BNV, BKV, TMV, TNV)                                                                  \
        do {                                                                                                \
            dim3 grid((unsigned)((d->n + BNV - 1) / BNV), (unsigned)((d->m + BMV - 1) / BMV), (unsigned)batch); \
            chai_gemm_simt<float, BMV, BNV, BKV, TMV, TNV><<<grid, (BMV / TMV) * (BNV / TNV), 0, ctx->stream>>>( \
                (const float*)d->a, (const float*)d->b, (float*)d->c, d->m, d->n, d->k, d->lda, d->ldb, d->ldc,  \
                (float)d->alpha, (float)d->beta, d->stride_a, d->stride_b, d->stride_c);                     \
        } while (0)
        if (tiles(128, 128) >= ctx->sm_count) CHAI_SIMT(128, 128, 8, 8, 8);
        else if (tiles(64, 64) >= ctx->sm_count) CHAI_SIMT(64, 64, 32, 4, 4);
        else CHAI_SIMT(32, 64, 32, 4, 4);                  // 128 threads, 4 x 4 outputs each
#undef CHAI_SIMT
    }
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    return CHAI_OK;
}

}  // namespace chai
