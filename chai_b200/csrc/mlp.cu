// The tuner's cost model: a 14 -> 128 -> 128 -> 128 -> 1 ReLU MLP mapping
// GEMM/GEMV shape and tile-configuration features to log(runtime).  Trained
// and served on the GPU by the kernels in this file: a shared-memory tiled
// FP32 matmul with optional transposes (forward and the backward input
// gradient), a split-K form for the weight and bias gradients (K = samples),
// bias / ReLU, mean-squared-error gradient and Adam.  The reference's counterpart is the EM search of
// autotune/StandardEM.cpp:69-147, which has no model: it times every
// candidate.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "internal.h"
#include "mlp.h"

namespace chai {

// C[M x N] = op(A) op(B) (+ C when acc), op = transpose when t* != 0;
// A is M x K (or K x M transposed), B is K x N (or N x K).  16 x 16 tiles.
__global__ void mlp_matmul(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C, int M,
                           int N, int K, int ta, int tb, int acc)
{
    __shared__ float as[16][17], bs[16][17];
    const int r = blockIdx.y * 16 + threadIdx.y, c = blockIdx.x * 16 + threadIdx.x;
    float sum = 0.0f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
        as[threadIdx.y][threadIdx.x] = (r < M && ka < K) ? (ta ? A[(long long)ka * M + r] : A[(long long)r * K + ka]) : 0.0f;
        bs[threadIdx.y][threadIdx.x] = (kb < K && c < N) ? (tb ? B[(long long)c * K + kb] : B[(long long)kb * N + c]) : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; k++) sum = fmaf(as[threadIdx.y][k], bs[k][threadIdx.x], sum);
        __syncthreads();
    }
    if (r < M && c < N) C[(long long)r * N + c] = acc ? C[(long long)r * N + c] + sum : sum;
}

// Split-K product for the gradients, whose K is the sample count (10^5 and
// more for a full training set): block z covers k in [z kc, (z + 1) kc) and
// writes its partial C to P + z M N; mlp_splitk_sum adds the partials in a
// fixed order, so the gradients are deterministic.
__global__ void mlp_matmul_splitk(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ P,
                                  int M, int N, int K, int kc, int ta, int tb)
{
    __shared__ float as[16][17], bs[16][17];
    const int r = blockIdx.y * 16 + threadIdx.y, c = blockIdx.x * 16 + threadIdx.x;
    const int kbeg = blockIdx.z * kc, kend = min(K, kbeg + kc);
    float sum = 0.0f;
    for (int k0 = kbeg; k0 < kend; k0 += 16) {
        const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
        as[threadIdx.y][threadIdx.x] = (r < M && ka < kend) ? (ta ? A[(long long)ka * M + r] : A[(long long)r * K + ka]) : 0.0f;
        bs[threadIdx.y][threadIdx.x] = (kb < kend && c < N) ? (tb ? B[(long long)c * K + kb] : B[(long long)kb * N + c]) : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; k++) sum = fmaf(as[threadIdx.y][k], bs[k][threadIdx.x], sum);
        __syncthreads();
    }
    if (r < M && c < N) P[(long long)blockIdx.z * M * N + (long long)r * N + c] = sum;
}

__global__ void mlp_splitk_sum(const float* __restrict__ P, float* __restrict__ C, int splits, int mn)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= mn) return;
    float s = 0.0f;
    for (int z = 0; z < splits; z++) s += P[(long long)z * mn + i];
    C[i] = s;
}

__global__ void mlp_fill(float* __restrict__ p, long long n, float v)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void mlp_bias_act(float* __restrict__ Y, const float* __restrict__ b, long long M, int N, int relu)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= M * N) return;
    float v = Y[i] + b[i % N];
    Y[i] = relu ? fmaxf(v, 0.0f) : v;
}

__global__ void mlp_relu_back(float* __restrict__ dY, const float* __restrict__ Y, long long n)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i < n && Y[i] <= 0.0f) dY[i] = 0.0f;
}

// d = 2 (p - y) / n; per-block partial of the squared error (deterministic)
__global__ void mlp_mse(const float* __restrict__ p, const float* __restrict__ y, float* __restrict__ d,
                        double* __restrict__ part, long long n)
{
    __shared__ double sm[256];
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    double e = 0.0;
    if (i < n) {
        const float diff = p[i] - y[i];
        d[i] = 2.0f * diff / (float)n;
        e = (double)diff * diff;
    }
    sm[threadIdx.x] = e;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

__global__ void mlp_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                         float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Inference: the whole network for one sample per CTA in one launch (thread j
// owns hidden unit j; activations stay in shared memory).  Each dot product
// runs from zero over the inputs in order and adds the bias last, the same
// order as the layered training forward pass, so both give identical results.
__global__ void __launch_bounds__(MLP_H) mlp_infer(const float* __restrict__ params, const float* __restrict__ x,
                                                   float* __restrict__ out, int n, int w1, int b1, int w2, int b2,
                                                   int w3, int b3, int w4, int b4)
{
    __shared__ float h0[MLP_H], h1[MLP_H], xin[MLP_IN];
    const int s = blockIdx.x, j = threadIdx.x;
    if (s >= n) return;
    if (j < MLP_IN) xin[j] = x[(long long)s * MLP_IN + j];
    __syncthreads();
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) acc = fmaf(xin[i], __ldg(params + w1 + i * MLP_H + j), acc);
    h0[j] = fmaxf(acc + __ldg(params + b1 + j), 0.0f);
    __syncthreads();
    acc = 0.0f;
#pragma unroll 8
    for (int i = 0; i < MLP_H; i++) acc = fmaf(h0[i], __ldg(params + w2 + i * MLP_H + j), acc);
    h1[j] = fmaxf(acc + __ldg(params + b2 + j), 0.0f);
    __syncthreads();
    acc = 0.0f;
#pragma unroll 8
    for (int i = 0; i < MLP_H; i++) acc = fmaf(h1[i], __ldg(params + w3 + i * MLP_H + j), acc);
    __syncthreads();
    h0[j] = fmaxf(acc + __ldg(params + b3 + j), 0.0f);
    __syncthreads();
    if (j == 0) {
        acc = 0.0f;
        for (int i = 0; i < MLP_H; i++) acc = fmaf(h0[i], __ldg(params + w4 + i), acc);
        out[s] = acc + __ldg(params + b4);
    }
}

static unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

Mlp::Mlp(chai_cuda_ctx* ctx) : ctx_(ctx)
{
    const int dims[5] = {MLP_IN, MLP_H, MLP_H, MLP_H, 1};
    size_t off = 0;
    for (int l = 0; l < 4; l++) {
        in_[l] = dims[l];
        out_[l] = dims[l + 1];
        w_off_[l] = off;
        off += (size_t)dims[l] * dims[l + 1];
        b_off_[l] = off;
        off += dims[l + 1];
    }
    count_ = off;
}

Mlp::~Mlp()
{
    for (float* p : {params_, grads_, m_, v_}) if (p) cudaFree(p);
    for (float* p : acts_) if (p) cudaFree(p);
    for (float* p : dacts_) if (p) cudaFree(p);
    if (x_) cudaFree(x_);
    if (y_) cudaFree(y_);
    if (part_) cudaFree(part_);
    if (splitk_) cudaFree(splitk_);
    if (ones_) cudaFree(ones_);
    if (host_) cudaFreeHost(host_);
}

int Mlp::ensure(size_t n)
{
    if (!params_) {
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&params_, count_ * sizeof(float)));
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&grads_, count_ * sizeof(float)));
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&m_, count_ * sizeof(float)));
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&v_, count_ * sizeof(float)));
        init(1);
    }
    if (n <= cap_) return CHAI_OK;
    for (float*& p : acts_) { if (p) cudaFree(p); p = nullptr; }
    for (float*& p : dacts_) { if (p) cudaFree(p); p = nullptr; }
    if (x_) cudaFree(x_);
    if (y_) cudaFree(y_);
    if (part_) cudaFree(part_);
    if (ones_) cudaFree(ones_);
    ones_ = nullptr;
    if (!splitk_) CHAI_CUDA_TRY(ctx_, cudaMalloc(&splitk_, (size_t)kMaxSplits * MLP_H * MLP_H * sizeof(float)));
    for (int l = 0; l < 4; l++) {
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&acts_[l], n * out_[l] * sizeof(float)));
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&dacts_[l], n * out_[l] * sizeof(float)));
    }
    CHAI_CUDA_TRY(ctx_, cudaMalloc(&x_, n * MLP_IN * sizeof(float)));
    CHAI_CUDA_TRY(ctx_, cudaMalloc(&y_, n * sizeof(float)));
    CHAI_CUDA_TRY(ctx_, cudaMalloc(&part_, blocks_for((long long)n) * sizeof(double)));
    CHAI_CUDA_TRY(ctx_, cudaMalloc(&ones_, n * sizeof(float)));
    mlp_fill<<<blocks_for((long long)n), 256, 0, ctx_->stream>>>(ones_, (long long)n, 1.0f);
    cap_ = n;
    return CHAI_OK;
}

// He-uniform weights, zero biases (host RNG, seeded)
void Mlp::init(uint64_t seed)
{
    std::vector<float> h(count_, 0.0f);
    std::mt19937_64 g(seed);
    for (int l = 0; l < 4; l++) {
        const float lim = std::sqrt(6.0f / (float)in_[l]);
        std::uniform_real_distribution<float> u(-lim, lim);
        for (size_t i = 0; i < (size_t)in_[l] * out_[l]; i++) h[w_off_[l] + i] = u(g);
    }
    cudaMemcpy(params_, h.data(), count_ * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(m_, 0, count_ * sizeof(float));
    cudaMemset(v_, 0, count_ * sizeof(float));
    step_ = 0;
}

int Mlp::upload(const float* x, const float* y, size_t n)
{
    int st = ensure(n);
    if (st) return st;
    CHAI_CUDA_TRY(ctx_, cudaMemcpyAsync(x_, x, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, ctx_->stream));
    if (y) CHAI_CUDA_TRY(ctx_, cudaMemcpyAsync(y_, y, n * sizeof(float), cudaMemcpyHostToDevice, ctx_->stream));
    return CHAI_OK;
}

void Mlp::forward(size_t n)
{
    cudaStream_t s = ctx_->stream;
    const float* in = x_;
    for (int l = 0; l < 4; l++) {
        dim3 grid((out_[l] + 15) / 16, (unsigned)((n + 15) / 16));
        mlp_matmul<<<grid, dim3(16, 16), 0, s>>>(in, params_ + w_off_[l], acts_[l], (int)n, out_[l], in_[l], 0, 0, 0);
        mlp_bias_act<<<blocks_for((long long)n * out_[l]), 256, 0, s>>>(acts_[l], params_ + b_off_[l], (long long)n,
                                                                         out_[l], l < 3);
        in = acts_[l];
    }
}

double Mlp::backward(size_t n)
{
    cudaStream_t s = ctx_->stream;
    const unsigned nb = blocks_for((long long)n);
    mlp_mse<<<nb, 256, 0, s>>>(acts_[3], y_, dacts_[3], part_, (long long)n);
    for (int l = 3; l >= 0; l--) {
        if (l < 3) mlp_relu_back<<<blocks_for((long long)n * out_[l]), 256, 0, s>>>(dacts_[l], acts_[l], (long long)n * out_[l]);
        const float* in = l == 0 ? x_ : acts_[l - 1];
        // dW = in^T dY  (in_[l] x out_[l]) and db = 1^T dY, split over the samples
        splitk(in, dacts_[l], grads_ + w_off_[l], in_[l], out_[l], n);
        splitk(ones_, dacts_[l], grads_ + b_off_[l], 1, out_[l], n);
        if (l > 0) {
            // dX = dY W^T  (n x in_[l])
            dim3 gx((in_[l] + 15) / 16, (unsigned)((n + 15) / 16));
            mlp_matmul<<<gx, dim3(16, 16), 0, s>>>(dacts_[l], params_ + w_off_[l], dacts_[l - 1], (int)n, in_[l],
                                                   out_[l], 0, 1, 0);
        }
    }
    std::vector<double> part(nb);
    cudaMemcpyAsync(part.data(), part_, nb * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double e = 0.0;
    for (double v : part) e += v;
    return e / (double)n;
}

// C (M x N) = A^T B over K = n samples (A: n x M, B: n x N), split over K
void Mlp::splitk(const float* A, const float* B, float* C, int M, int N, size_t n)
{
    cudaStream_t s = ctx_->stream;
    const int kc = std::max(256, (int)(((n + kMaxSplits - 1) / kMaxSplits + 15) / 16 * 16));
    const int splits = (int)((n + kc - 1) / kc);
    dim3 g((N + 15) / 16, (M + 15) / 16, (unsigned)splits);
    mlp_matmul_splitk<<<g, dim3(16, 16), 0, s>>>(A, B, splitk_, M, N, (int)n, kc, 1, 0);
    mlp_splitk_sum<<<(M * N + 255) / 256, 256, 0, s>>>(splitk_, C, splits, M * N);
}

void Mlp::adam(double lr)
{
    step_++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)step_), c2 = 1.0f - std::pow(b2, (float)step_);
    mlp_adam<<<blocks_for((long long)count_), 256, 0, ctx_->stream>>>(params_, grads_, m_, v_, (long long)count_,
                                                                       (float)lr, b1, b2, 1e-8f, c1, c2);
}

// Targets are standardised (y - mean) / scale; predictions are mapped back.
int Mlp::train(const std::vector<float>& x, const std::vector<float>& y_raw, int epochs, double lr, uint64_t seed,
               double* loss)
{
    const size_t n = y_raw.size();
    if (n == 0) return set_error(ctx_, CHAI_ERR_INVALID, "mlp: no samples");
    double mu = 0, var = 0;
    for (float v : y_raw) mu += v;
    mu /= (double)n;
    for (float v : y_raw) var += (v - mu) * (v - mu);
    mean_ = (float)mu;
    scale_ = (float)std::sqrt(var / (double)n + 1e-12);
    std::vector<float> y(n);
    for (size_t i = 0; i < n; i++) y[i] = (y_raw[i] - mean_) / scale_;
    int st = ensure(n);
    if (st) return st;
    init(seed);
    st = upload(x.data(), y.data(), n);
    if (st) return st;
    double l = 0;
    for (int e = 0; e < epochs; e++) {
        forward(n);
        l = backward(n);
        adam(lr);
    }
    trained_ = true;
    if (loss) *loss = l;
    CHAI_CUDA_TRY(ctx_, cudaStreamSynchronize(ctx_->stream));
    return CHAI_OK;
}

int Mlp::predict(const std::vector<float>& x, std::vector<double>& out)
{
    const size_t n = x.size() / MLP_IN;
    out.resize(n);
    if (n == 0) return CHAI_OK;
    int st = ensure(n);
    if (st) return st;
    if (n > host_cap_) {
        if (host_) cudaFreeHost(host_);
        host_ = nullptr;
        host_cap_ = 0;
        CHAI_CUDA_TRY(ctx_, cudaMallocHost(&host_, n * (MLP_IN + 1) * sizeof(float)));
        host_cap_ = n;
    }
    float* hx = host_;
    float* hp = host_ + n * MLP_IN;
    std::copy(x.begin(), x.end(), hx);
    cudaStream_t s = ctx_->stream;
    CHAI_CUDA_TRY(ctx_, cudaMemcpyAsync(x_, hx, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, s));
    mlp_infer<<<(unsigned)n, MLP_H, 0, s>>>(params_, x_, acts_[3], (int)n, (int)w_off_[0], (int)b_off_[0],
                                             (int)w_off_[1], (int)b_off_[1], (int)w_off_[2], (int)b_off_[2],
                                             (int)w_off_[3], (int)b_off_[3]);
    CHAI_CUDA_TRY(ctx_, cudaGetLastError());
    CHAI_CUDA_TRY(ctx_, cudaMemcpyAsync(hp, acts_[3], n * sizeof(float), cudaMemcpyDeviceToHost, s));
    CHAI_CUDA_TRY(ctx_, cudaStreamSynchronize(s));
    for (size_t i = 0; i < n; i++) out[i] = (double)hp[i] * scale_ + mean_;
    return CHAI_OK;
}

int Mlp::gradients(const std::vector<float>& x, const std::vector<float>& y_raw, std::vector<float>& g, double* loss)
{
    const size_t n = y_raw.size();
    std::vector<float> y(n);
    for (size_t i = 0; i < n; i++) y[i] = (y_raw[i] - mean_) / scale_;
    int st = upload(x.data(), y.data(), n);
    if (st) return st;
    forward(n);
    const double l = backward(n);
    g.resize(count_);
    CHAI_CUDA_TRY(ctx_, cudaMemcpy(g.data(), grads_, count_ * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return CHAI_OK;
}

int Mlp::weights(float* buf, size_t cap, size_t* count, int set)
{
    int st = ensure(1);
    if (st) return st;
    if (count) *count = count_ + 2;
    if (!buf) return CHAI_OK;
    if (cap < count_ + 2) return set_error(ctx_, CHAI_ERR_INVALID, "mlp weights: buffer too small");
    if (set) {
        CHAI_CUDA_TRY(ctx_, cudaMemcpy(params_, buf, count_ * sizeof(float), cudaMemcpyHostToDevice));
        mean_ = buf[count_];
        scale_ = buf[count_ + 1];
        trained_ = true;
    } else {
        CHAI_CUDA_TRY(ctx_, cudaMemcpy(buf, params_, count_ * sizeof(float), cudaMemcpyDeviceToHost));
        buf[count_] = mean_;
        buf[count_ + 1] = scale_;
    }
    return CHAI_OK;
}

}  // namespace chai
