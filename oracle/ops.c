/* CPU restatement of the reference interpreter's deterministic array ops
 * (the oracle for matmul, GEMV, reductions and gather).  Test infrastructure
 * only: tests, the smoke check and the bench's CPU baseline call this; the
 * product never links it.
 *
 * Semantics followed:
 *   matmul / GEMM   interp/InterpMatmulBase.hpp:25-61 (row-major, result
 *                   width = B's width, height = A's height; f32 products
 *                   accumulated in double: oracle_matmul_ref_f32; GEMM
 *                   C = alpha*AB + beta*C)
 *   matvec          interp/InterpMatmulBase.hpp:37-47
 *   sum / mean / dot_product   interp/InterpAccum.cpp:13-70,
 *                   interp/InterpDotprod.cpp:14-60 (double accumulator)
 *   gather2_floor   interp/InterpGather.hpp:19-44 (floor index, add W if
 *                   negative, modulo W: periodic wrap)
 * The double GEMM is blocked and OpenMP-parallel: it is the FP64 accuracy
 * oracle for GEMM shapes the single-threaded interpreter cannot finish. */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* C[M][N] = sum_k A[M][K] * B[K][N] in double, inputs f32 */
void oracle_gemm_f32_to_f64(int64_t M, int64_t N, int64_t K, const float* A, const float* B, double* C)
{
    const int64_t BK = 256, BN = 512;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < M; i++) {
        double* c = C + i * N;
        for (int64_t j = 0; j < N; j++) c[j] = 0.0;
        for (int64_t k0 = 0; k0 < K; k0 += BK) {
            const int64_t k1 = k0 + BK < K ? k0 + BK : K;
            for (int64_t j0 = 0; j0 < N; j0 += BN) {
                const int64_t j1 = j0 + BN < N ? j0 + BN : N;
                for (int64_t k = k0; k < k1; k++) {
                    const double a = (double)A[i * K + k];
                    const float* b = B + k * N;
                    for (int64_t j = j0; j < j1; j++) c[j] += a * (double)b[j];
                }
            }
        }
    }
}

/* The interpreter's matmul arithmetic (interp/InterpMatmulBase.hpp:50-61):
 * each product of two f32 operands is rounded to f32, then accumulated in
 * double with k ascending; the f32 result is the double sum rounded.  When the
 * inner dimensions differ the interpreter wraps both (z % K_a, z % K_b) up to
 * the larger one. */
void oracle_matmul_ref_f32(int64_t M, int64_t N, int64_t Ka, int64_t Kb, const float* A, const float* B, float* C)
{
    const int64_t K = Ka > Kb ? Ka : Kb;
    #pragma omp parallel for
    for (int64_t i = 0; i < M; i++)
        for (int64_t j = 0; j < N; j++) {
            double acc = 0.0;
            for (int64_t z = 0; z < K; z++) {
                const float p = A[i * Ka + z % Ka] * B[(z % Kb) * N + j];
                acc += (double)p;
            }
            C[i * N + j] = (float)acc;
        }
}

/* matrix-vector with the same arithmetic (InterpMatmulBase.hpp:37-47) */
void oracle_matvec_ref_f32(int64_t M, int64_t Na, int64_t Nx, const float* A, const float* x, float* y)
{
    const int64_t N = Na > Nx ? Na : Nx;
    #pragma omp parallel for
    for (int64_t i = 0; i < M; i++) {
        double acc = 0.0;
        for (int64_t z = 0; z < N; z++) {
            const float p = A[i * Na + z % Na] * x[z % Nx];
            acc += (double)p;
        }
        y[i] = (float)acc;
    }
}

/* a subset of entries of C = A B (rows[i], cols[i]) in double */
void oracle_gemm_entries_f64(int64_t N, int64_t K, const float* A, const float* B,
                             int64_t n_entries, const int64_t* rows, const int64_t* cols, double* out)
{
    #pragma omp parallel for
    for (int64_t e = 0; e < n_entries; e++) {
        const float* a = A + rows[e] * K;
        double acc = 0.0;
        for (int64_t k = 0; k < K; k++) acc += (double)a[k] * (double)B[k * N + cols[e]];
        out[e] = acc;
    }
}

/* y[M] = A[M][N] x[N], double accumulation, f64 or f32 storage */
void oracle_gemv_f64(int64_t M, int64_t N, const double* A, const double* x, double* y)
{
    #pragma omp parallel for
    for (int64_t i = 0; i < M; i++) {
        double acc = 0.0;
        for (int64_t j = 0; j < N; j++) acc += A[i * N + j] * x[j];
        y[i] = acc;
    }
}

void oracle_gemv_f32(int64_t M, int64_t N, const float* A, const float* x, double* y)
{
    #pragma omp parallel for
    for (int64_t i = 0; i < M; i++) {
        double acc = 0.0;
        for (int64_t j = 0; j < N; j++) acc += (double)A[i * N + j] * (double)x[j];
        y[i] = acc;
    }
}

/* sum in double, sequential order as the interpreter loops */
double oracle_sum_f32(int64_t n, const float* a)
{
    double acc = 0.0;
    for (int64_t i = 0; i < n; i++) acc += (double)a[i];
    return acc;
}

/* dot_product of two f32 arrays as interp/InterpDotprod.cpp:14-60 computes
 * it: each product in f32 (float * float), accumulated in double */
double oracle_dot_f32(int64_t n, const float* a, const float* b)
{
    double acc = 0.0;
    for (int64_t i = 0; i < n; i++) {
        const float p = a[i] * b[i];
        acc += (double)p;
    }
    return acc;
}

/* periodic index wrap of gather2_floor */
static inline int64_t wrap_idx(double v, int64_t n)
{
    int64_t i = (int64_t)floor(v);
    i %= n;
    if (i < 0) i += n;
    return i;
}

/* out[y][x] = A[wrap(floor(Y))][wrap(floor(X))] */
void oracle_gather2_floor_f32(int64_t W, int64_t H, const float* A, const float* X, const float* Y, float* out)
{
    #pragma omp parallel for
    for (int64_t y = 0; y < H; y++)
        for (int64_t x = 0; x < W; x++) {
            const int64_t i = y * W + x;
            out[i] = A[wrap_idx(Y[i], H) * W + wrap_idx(X[i], W)];
        }
}

/* 8-direction Kirsch compass response: each mask weighs three consecutive
 * neighbours (clockwise from north-west) by 5 and the other five by -3; the
 * output is the maximum response.  Evaluated as the traced program does:
 * r_k = 8*(n_k + n_k+1 + n_k+2) - 3*total, in f32, left to right. */
void oracle_kirsch_f32(int64_t W, int64_t H, const float* A, float* out)
{
    static const int dx[8] = {-1, 0, 1, 1, 1, 0, -1, -1};
    static const int dy[8] = {-1, -1, -1, 0, 1, 1, 1, 0};
    #pragma omp parallel for
    for (int64_t y = 0; y < H; y++)
        for (int64_t x = 0; x < W; x++) {
            float n[8];
            for (int k = 0; k < 8; k++) {
                int64_t yy = (y + dy[k]) % H; if (yy < 0) yy += H;
                int64_t xx = (x + dx[k]) % W; if (xx < 0) xx += W;
                n[k] = A[yy * W + xx];
            }
            float total = n[0];
            for (int k = 1; k < 8; k++) total = total + n[k];
            float best = -INFINITY;
            for (int k = 0; k < 8; k++) {
                float three = (n[k] + n[(k + 1) % 8]) + n[(k + 2) % 8];
                float r = 8.0f * three - 3.0f * total;
                if (r > best) best = r;
            }
            out[y * W + x] = best;
        }
}
