// Cost-model MLP of the tuner (mlp.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "tuner.h"

struct chai_cuda_ctx;

namespace chai {

class Mlp {
public:
    explicit Mlp(chai_cuda_ctx* ctx);
    ~Mlp();
    // x: n x MLP_IN row-major features; y: log(runtime in us)
    int train(const std::vector<float>& x, const std::vector<float>& y, int epochs, double lr, uint64_t seed,
              double* loss);
    int predict(const std::vector<float>& x, std::vector<double>& out);
    int gradients(const std::vector<float>& x, const std::vector<float>& y, std::vector<float>& g, double* loss);
    int weights(float* buf, size_t cap, size_t* count, int set);
    bool trained() const { return trained_; }

private:
    chai_cuda_ctx* ctx_;
    int in_[4], out_[4];
    size_t w_off_[4], b_off_[4], count_ = 0;
    float* params_ = nullptr;
    float* grads_ = nullptr;
    float* m_ = nullptr;
    float* v_ = nullptr;
    float* acts_[4] = {nullptr, nullptr, nullptr, nullptr};
    float* dacts_[4] = {nullptr, nullptr, nullptr, nullptr};
    float* x_ = nullptr;
    float* y_ = nullptr;
    double* part_ = nullptr;
    float* splitk_ = nullptr;            // split-K partial gradients (kMaxSplits x MLP_H x MLP_H)
    float* ones_ = nullptr;              // n ones: the bias gradient is 1^T dY
    static constexpr int kMaxSplits = 64;
    float* host_ = nullptr;              // pinned staging of inference inputs / outputs
    size_t host_cap_ = 0;
    size_t cap_ = 0;
    long long step_ = 0;
    float mean_ = 0.0f, scale_ = 1.0f;
    bool trained_ = false;
    int ensure(size_t n);
    void init(uint64_t seed);
    int upload(const float* x, const float* y, size_t n);
    void forward(size_t n);
    double backward(size_t n);
    void adam(double lr);
    void splitk(const float* A, const float* B, float* C, int M, int N, size_t n);
};

}  // namespace chai
