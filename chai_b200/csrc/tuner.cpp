// GEMM / GEMV tuner: exhaustive sweep ("AutoTuneBench"), learned top-k ranking
// with the MLP cost model, tuning DB and crash-safe journal.
//
// Reference counterparts: StandardEM::searchLoop / timingLoop
// (autotune/StandardEM.cpp:69-147) alternate coordinate searches over
// work-group size, inner blocking and extra parameters and time one launch
// per candidate with gettimeofday (autotune/AutoTuneBench.cpp:17-251); the
// journal marks each risky step so a crash marks the kernel bad on restart
// (autotune/AutoTuneMemo.hpp:20-28).  Here the search space is the tile
// configuration of this library's own kernels (tuner.h) and every timing uses
// CUDA events on the context stream.  The exhaustive sweep times each
// configuration as one warm-up launch plus the best of 3; the learned mode
// ranks all configurations with the MLP and times only the top k, one launch
// each (k = 1: no timing at all).  Every kernel variant is loaded before the
// first timing, so no timed launch includes module loading.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "internal.h"
#include "mlp.h"
#include "tuner.h"

namespace chai {

static std::tuple<long long, long long, long long, int, int> key_of(const chai_gemm_key& k)
{
    return std::make_tuple((long long)k.m, (long long)k.n, (long long)k.is_gemv ? 1ll : (long long)k.k,
                           (int)k.precision, (int)k.is_gemv);
}

static std::string key_str(const chai_gemm_key& k, const chai_gemm_cfg& c)
{
    std::ostringstream os;
    os << k.m << ' ' << k.n << ' ' << (k.is_gemv ? 1 : k.k) << ' ' << k.precision << ' ' << k.is_gemv << ' '
       << c.block_m << ' ' << c.block_n << ' ' << c.block_k << ' ' << c.stages << ' ' << c.vec_width << ' '
       << c.cluster_m << ' ' << c.cluster_n << ' ' << c.group_m;
    return os.str();
}

Tuner::Tuner(chai_cuda_ctx* ctx) : ctx_(ctx), mlp_(new Mlp(ctx))
{
    journal_ = ctx->cfg.tune_journal;
    top_k = ctx->cfg.top_k;
}

Tuner::~Tuner()
{
    delete mlp_;
    for (void* p : bufs_) if (p) cudaFree(p);
}

std::vector<chai_gemm_cfg> Tuner::space(const chai_gemm_key& key)
{
    std::vector<chai_gemm_cfg> v;
    if (key.is_gemv) {
        chai_gemm_cfg bulk{};          // warps 0: the cp.async.bulk kernel
        bulk.vec_width = 1;
        bulk.cluster_m = bulk.cluster_n = 1;
        v.push_back(bulk);
        for (int w : {2, 4, 8, 16})
            for (int u : {1, 2, 4, 8}) {
                chai_gemm_cfg c{};
                c.block_m = w;
                c.vec_width = u;
                c.cluster_m = c.cluster_n = 1;
                v.push_back(c);
            }
        return v;
    }
    // one-CTA tiles (block_m 128): N tile 64 / 128 / 256 with their stage
    // counts; CTA-pair tiles (block_m 256, cluster 2 x 1): N tile 128 / 256;
    // each over eight tile-raster group heights
    struct Tile { int bm, bn, stages; };
    static const Tile tiles[] = {{128, 64, 4}, {128, 64, 6}, {128, 64, 8}, {128, 128, 4}, {128, 128, 6},
                                 {128, 256, 3}, {128, 256, 4}, {256, 128, 4}, {256, 128, 6}, {256, 128, 8},
                                 {256, 256, 3}, {256, 256, 4}, {256, 256, 6}};
    for (const Tile& t : tiles)
        for (int g : {1, 2, 4, 8, 16, 32, 64, 128}) {
            chai_gemm_cfg c{};
            c.block_m = t.bm;
            c.block_n = t.bn;
            c.block_k = 128;
            c.stages = t.stages;
            c.vec_width = 4;
            c.cluster_m = t.bm == 256 ? 2 : 1;
            c.cluster_n = 1;
            c.group_m = g;
            v.push_back(c);
        }
    return v;
}

// Fraction of the last wave of work units that has work: GEMM tiles of
// block_m x block_n over a persistent grid (148 one-CTA tiles or 74 CTA pairs
// at a time); GEMV blocks of `warps` rows with 64 / warps blocks per SM.
static double wave_efficiency(const chai_gemm_key& key, const chai_gemm_cfg& c)
{
    const double sms = 148.0;
    double units, per_wave;
    if (key.is_gemv) {
        const int w = std::max(1, c.block_m);
        units = std::ceil((double)std::max<long long>(1, key.m) / w);
        per_wave = sms * std::max(1, std::min(32, 64 / w));
    } else {
        const int bm = c.block_m == 256 ? 256 : 128, bn = std::max(1, c.block_n);
        units = std::ceil((double)std::max<long long>(1, key.m) / bm) *
                std::ceil((double)std::max<long long>(1, key.n) / bn);
        per_wave = bm == 256 ? sms / 2 : sms;
    }
    return units / (std::ceil(units / per_wave) * per_wave);
}

// Fraction of the tiles' area inside the product (tile quantisation)
static double tile_fill(const chai_gemm_key& key, const chai_gemm_cfg& c)
{
    if (key.is_gemv) return 0.0;
    const double m = std::max<long long>(1, key.m), n = std::max<long long>(1, key.n);
    const double bm = c.block_m == 256 ? 256 : 128, bn = std::max(1, c.block_n);
    return (m * n) / (std::ceil(m / bm) * bm * std::ceil(n / bn) * bn);
}

void Tuner::features(const chai_gemm_key& key, const chai_gemm_cfg& c, float* f)
{
    const double m = std::max<long long>(1, key.m), n = std::max<long long>(1, key.n);
    const double k = key.is_gemv ? 1.0 : std::max<long long>(1, key.k);
    const bool split = key.precision == CHAI_GEMM_BF16X3 || key.precision == CHAI_GEMM_BF16X6 ||
                       key.precision == CHAI_GEMM_FP32;
    f[0] = (float)(std::log2(m) / 14.0);
    f[1] = (float)(std::log2(n) / 14.0);
    f[2] = (float)(std::log2(k) / 14.0);
    f[3] = !key.is_gemv && split ? 1.0f : 0.0f;
    f[4] = !key.is_gemv && !split ? 1.0f : 0.0f;
    f[5] = key.is_gemv ? 1.0f : 0.0f;
    f[6] = !key.is_gemv && c.block_m == 256 ? 1.0f : 0.0f;
    f[7] = (float)c.block_n / 256.0f;
    f[8] = (float)c.stages / 8.0f;
    f[9] = c.group_m > 0 ? (float)(std::log2((double)c.group_m) / 7.0) : 0.0f;
    f[10] = key.is_gemv ? (float)c.block_m / 16.0f : 0.0f;
    f[11] = key.is_gemv ? (float)c.vec_width / 8.0f : 0.0f;
    f[12] = (float)wave_efficiency(key, c);
    f[13] = (float)tile_fill(key, c);
}

int Tuner::ensure_operands(const chai_gemm_key& key)
{
    const size_t eb = key.precision == CHAI_GEMM_FP64 ? 8 : 4;
    size_t need[3];
    if (key.is_gemv) {
        need[0] = (size_t)key.m * key.n * eb;
        need[1] = (size_t)key.n * eb;
        need[2] = (size_t)key.m * eb;
    } else {
        need[0] = (size_t)key.m * key.k * 4;
        need[1] = (size_t)key.k * key.n * 4;
        need[2] = (size_t)key.m * key.n * 4;
    }
    for (int i = 0; i < 3; i++) {
        if (buf_bytes_[i] >= need[i]) continue;
        if (bufs_[i]) cudaFree(bufs_[i]);
        bufs_[i] = nullptr;
        buf_bytes_[i] = 0;
        const size_t bytes = (need[i] + (need[i] >> 3) + 4095) & ~size_t(4095);
        CHAI_CUDA_TRY(ctx_, cudaMalloc(&bufs_[i], bytes));
        buf_bytes_[i] = bytes;
        // uniform[-1, 1) operands from the library's own generator
        chai_rng_desc d{};
        d.variant = CHAI_RNG_PHILOX;
        d.prec = CHAI_F32;
        d.vec_len = 4;
        d.seed = 17 + i;
        d.width = bytes / 16 * 4;
        d.height = 1;
        d.slots = 1;
        d.has_limits = 1;
        d.min_limit = -1.0;
        d.max_limit = 1.0;
        int st = launch_rng_fill(ctx_, &d, bufs_[i]);
        if (st) return st;
    }
    return CHAI_OK;
}

int Tuner::time_cfg(const chai_gemm_key& key, chai_gemm_cfg& c, int reps, bool warm)
{
    const std::string ks = key_str(key, c);
    if (bad_.count(ks)) {
        c.measured_us = 1e30;
        return CHAI_OK;
    }
    if (!preloaded_) {
        preload_gemm_kernels();
        preload_gemv_kernels();
        preloaded_ = true;
    }
    int st = ensure_operands(key);
    if (st) return st;
    if (!journal_.empty()) {
        std::ofstream j(journal_, std::ios::app);
        j << "TRY " << ks << "\n";
    }
    auto run = [&]() -> int {
        if (key.is_gemv) {
            GemvCfg g;
            g.warps = c.block_m;
            g.unroll = c.vec_width;
            return launch_gemv_cfg(ctx_, key.precision == CHAI_GEMM_FP64 ? CHAI_F64 : CHAI_F32, 0, key.m, key.n, 1.0,
                                   bufs_[0], key.n, bufs_[1], 0.0, bufs_[2], &g);
        }
        chai_gemm_desc d{};
        d.precision = key.precision == CHAI_GEMM_FP32 ? CHAI_GEMM_BF16X3 : key.precision;
        d.m = key.m;
        d.n = key.n;
        d.k = key.k;
        d.a = bufs_[0];
        d.lda = key.k;
        d.b = bufs_[1];
        d.ldb = key.n;
        d.c = bufs_[2];
        d.ldc = key.n;
        d.alpha = 1.0;
        d.beta = 0.0;
        d.batch = 1;
        TcCfg t;
        t.bm = c.block_m == 256 ? 256 : 128;
        t.bn = c.block_n;
        t.stages = c.stages;
        t.group_m = c.group_m;
        return launch_gemm_tc_cfg(ctx_, &d, d.precision, &t);
    };
    if (warm) {
        st = run();
        if (st) return st;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int r = 0; r < reps && !st; r++) {
        cudaEventRecord(e0, ctx_->stream);
        st = run();
        cudaEventRecord(e1, ctx_->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    c.measured_us = best * 1e3;
    if (!journal_.empty()) {
        std::ofstream j(journal_, std::ios::app);
        j << "OK " << ks << ' ' << c.measured_us << "\n";
    }
    return CHAI_OK;
}

int Tuner::sweep(const chai_gemm_key* key, chai_gemm_cfg* out, int cap, int* n)
{
    std::vector<chai_gemm_cfg> v = space(*key);
    if (n) *n = (int)v.size();
    for (size_t i = 0; i < v.size(); i++) {
        int st = time_cfg(*key, v[i], 3, true);
        if (st) return st;
        if (out && (int)i < cap) out[i] = v[i];
    }
    return CHAI_OK;
}

int Tuner::tune(const chai_gemm_key* key, int mode, chai_gemm_cfg* out)
{
    if (mode == CHAI_TUNE_DEFAULT) {
        // what an untuned call of this shape runs (GemvCfg / default_tc_cfg)
        chai_gemm_cfg c{};
        c.cluster_m = c.cluster_n = 1;
        if (key->is_gemv) {
            const GemvCfg g;
            c.block_m = g.warps;
            c.vec_width = g.unroll;
        } else {
            const TcCfg t = default_tc_cfg(key->m, key->n, ctx_->sm_count);
            c.block_m = t.bm;
            c.block_n = t.bn;
            c.block_k = 128;
            c.stages = t.stages;
            c.vec_width = 4;
            c.cluster_m = t.bm == 256 ? 2 : 1;
            c.group_m = t.group_m;
        }
        if (out) *out = c;
        return CHAI_OK;
    }
    std::vector<chai_gemm_cfg> v = space(*key);
    std::vector<chai_gemm_cfg> timed;
    if (mode == CHAI_TUNE_LEARNED && mlp_->trained()) {
        std::vector<float> x(v.size() * MLP_IN);
        for (size_t i = 0; i < v.size(); i++) features(*key, v[i], &x[i * MLP_IN]);
        std::vector<double> pred;
        int st = mlp_->predict(x, pred);
        if (st) return st;
        std::vector<size_t> order(v.size());
        for (size_t i = 0; i < order.size(); i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return pred[a] < pred[b]; });
        const size_t k = std::min<size_t>(std::max(1, top_k), v.size());
        for (size_t i = 0; i < k; i++) {
            chai_gemm_cfg c = v[order[i]];
            if (k > 1) {
                st = time_cfg(*key, c, 1, false);
                if (st) return st;
            } else {
                c.measured_us = std::exp(pred[order[i]]);
            }
            timed.push_back(c);
        }
    } else {
        for (auto& c : v) {
            int st = time_cfg(*key, c, 3, true);
            if (st) return st;
            timed.push_back(c);
        }
    }
    auto best = std::min_element(timed.begin(), timed.end(),
                                 [](const chai_gemm_cfg& a, const chai_gemm_cfg& b) { return a.measured_us < b.measured_us; });
    db_[key_of(*key)] = *best;
    if (out) *out = *best;
    return CHAI_OK;
}

bool Tuner::lookup(const chai_gemm_key* key, chai_gemm_cfg* out) const
{
    auto it = db_.find(key_of(*key));
    if (it == db_.end()) return false;
    if (out) *out = it->second;
    return true;
}

int Tuner::save(const std::string& path) const
{
    std::ofstream f(path);
    if (!f) return set_error(ctx_, CHAI_ERR_INVALID, "tune db: cannot write " + path);
    for (auto& kv : db_) {
        chai_gemm_key k{};
        k.m = std::get<0>(kv.first);
        k.n = std::get<1>(kv.first);
        k.k = std::get<2>(kv.first);
        k.precision = std::get<3>(kv.first);
        k.is_gemv = std::get<4>(kv.first);
        f << "BEST " << key_str(k, kv.second) << ' ' << kv.second.measured_us << "\n";
    }
    // MLP weights beside the DB
    size_t count = 0;
    mlp_->weights(nullptr, 0, &count, 0);
    if (mlp_->trained()) {
        std::vector<float> w(count);
        mlp_->weights(w.data(), w.size(), &count, 0);
        std::ofstream m(path + ".mlp", std::ios::binary);
        m.write(reinterpret_cast<const char*>(w.data()), (std::streamsize)(w.size() * sizeof(float)));
    }
    return CHAI_OK;
}

// DB lines: BEST <key> <cfg> <us>.  The journal (TuneJournal) is appended a
// TRY line before and an OK line after every timed configuration; a TRY with
// no OK means the process died while that configuration ran, and it is never
// timed again (autotune/AutoTuneMemo.hpp:20-28).
int Tuner::load(const std::string& path)
{
    if (!path.empty()) {
        std::ifstream f(path);
        std::string tag;
        while (f >> tag) {
            chai_gemm_key k{};
            chai_gemm_cfg c{};
            long long m = 0, n = 0, kk = 0;
            f >> m >> n >> kk >> k.precision >> k.is_gemv >> c.block_m >> c.block_n >> c.block_k >> c.stages >>
                c.vec_width >> c.cluster_m >> c.cluster_n >> c.group_m >> c.measured_us;
            if (!f) break;
            k.m = m;
            k.n = n;
            k.k = kk;
            if (tag == "BEST") db_[key_of(k)] = c;
        }
        std::ifstream w(path + ".mlp", std::ios::binary | std::ios::ate);
        if (w) {
            const size_t bytes = (size_t)w.tellg();
            w.seekg(0);
            std::vector<float> ws(bytes / sizeof(float));
            w.read(reinterpret_cast<char*>(ws.data()), (std::streamsize)(ws.size() * sizeof(float)));
            size_t count = 0;
            int st = mlp_->weights(nullptr, 0, &count, 0);
            if (st) return st;
            if (ws.size() == count) {
                st = mlp_->weights(ws.data(), ws.size(), &count, 1);
                if (st) return st;
            }
        }
    }
    if (!journal_.empty()) {
        std::ifstream j(journal_);
        std::string line;
        std::map<std::string, int> open;
        while (std::getline(j, line)) {
            if (line.rfind("TRY ", 0) == 0) {
                open[line.substr(4)]++;
            } else if (line.rfind("OK ", 0) == 0) {
                const std::string rest = line.substr(3, line.find_last_of(' ') - 3);
                if (open[rest] > 0) open[rest]--;
            }
        }
        for (auto& kv : open)
            if (kv.second > 0) bad_[kv.first] = 1;
    }
    return CHAI_OK;
}

bool tuned_tc_cfg(chai_cuda_ctx* ctx, long long m, long long n, long long k, int precision, TcCfg* out)
{
    if (!ctx->tuner) return false;
    chai_gemm_key key{};
    key.m = m;
    key.n = n;
    key.k = k;
    key.precision = precision;
    chai_gemm_cfg c;
    bool hit = ctx->tuner->lookup(&key, &c);
    if (!hit && precision == CHAI_GEMM_BF16X3) {   // tuned as "fp32" (split precision) keys
        key.precision = CHAI_GEMM_FP32;
        hit = ctx->tuner->lookup(&key, &c);
    }
    if (!hit) return false;
    out->bm = c.block_m == 256 ? 256 : 128;
    out->bn = c.block_n;
    out->stages = c.stages;
    out->group_m = c.group_m;
    return true;
}

bool tuned_gemv_cfg(chai_cuda_ctx* ctx, long long m, long long n, int prec, GemvCfg* out)
{
    if (!ctx->tuner) return false;
    chai_gemm_key key{};
    key.m = m;
    key.n = n;
    key.k = 1;
    key.precision = prec == CHAI_F64 ? CHAI_GEMM_FP64 : CHAI_GEMM_FP32;
    key.is_gemv = 1;
    chai_gemm_cfg c;
    if (!ctx->tuner->lookup(&key, &c)) return false;
    out->warps = c.block_m;
    out->unroll = c.vec_width;
    return true;
}

}  // namespace chai

using namespace chai;

static void samples(const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n, std::vector<float>& x,
                    std::vector<float>* y)
{
    x.resize(n * MLP_IN);
    if (y) y->resize(n);
    for (size_t i = 0; i < n; i++) {
        Tuner::features(keys[i], cfgs[i], &x[i * MLP_IN]);
        if (y) (*y)[i] = (float)std::log(std::max(cfgs[i].measured_us, 1e-3));
    }
}

static bool valid_key(const chai_gemm_key* k)
{
    if (k->m <= 0 || k->n <= 0 || (!k->is_gemv && k->k <= 0)) return false;
    if (k->is_gemv) return k->precision == CHAI_GEMM_FP32 || k->precision == CHAI_GEMM_FP64;
    return k->precision == CHAI_GEMM_FP32 || k->precision == CHAI_GEMM_TF32 || k->precision == CHAI_GEMM_BF16 ||
           k->precision == CHAI_GEMM_BF16X3 || k->precision == CHAI_GEMM_BF16X6;
}

extern "C" {

int chai_cuda_tune(chai_cuda_ctx* ctx, const chai_gemm_key* key, int mode, chai_gemm_cfg* out)
{
    if (!ctx || !key || !out) return CHAI_ERR_INVALID;
    if (!valid_key(key)) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "tune: shape or precision");
    return ctx->tuner->tune(key, mode, out);
}

int chai_cuda_tune_sweep(chai_cuda_ctx* ctx, const chai_gemm_key* key, chai_gemm_cfg* out, int cap, int* n)
{
    if (!ctx || !key) return CHAI_ERR_INVALID;
    if (!valid_key(key)) return set_error(ctx, CHAI_ERR_UNSUPPORTED, "tune: shape or precision");
    return ctx->tuner->sweep(key, out, cap, n);
}

int chai_cuda_tune_features(const chai_gemm_key* key, const chai_gemm_cfg* cfg, float* out)
{
    if (!key || !cfg || !out) return CHAI_ERR_INVALID;
    Tuner::features(*key, *cfg, out);
    return CHAI_OK;
}

int chai_cuda_tune_db_load(chai_cuda_ctx* ctx, const char* path)
{
    if (!ctx || !path) return CHAI_ERR_INVALID;
    return ctx->tuner->load(path);
}

int chai_cuda_tune_db_save(chai_cuda_ctx* ctx, const char* path)
{
    if (!ctx || !path) return CHAI_ERR_INVALID;
    return ctx->tuner->save(path);
}

int chai_cuda_mlp_train(chai_cuda_ctx* ctx, const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n,
                        int epochs, double lr, uint64_t seed, double* final_loss)
{
    if (!ctx || !keys || !cfgs || n == 0 || epochs < 0) return CHAI_ERR_INVALID;
    std::vector<float> x, y;
    samples(keys, cfgs, n, x, &y);
    return ctx->tuner->mlp()->train(x, y, epochs, lr, seed, final_loss);
}

int chai_cuda_mlp_predict(chai_cuda_ctx* ctx, const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n,
                          double* log_us)
{
    if (!ctx || !keys || !cfgs || !log_us) return CHAI_ERR_INVALID;
    std::vector<float> x;
    samples(keys, cfgs, n, x, nullptr);
    std::vector<double> p;
    int st = ctx->tuner->mlp()->predict(x, p);
    if (st) return st;
    for (size_t i = 0; i < n; i++) log_us[i] = p[i];
    return CHAI_OK;
}

int chai_cuda_mlp_gradients(chai_cuda_ctx* ctx, const chai_gemm_key* keys, const chai_gemm_cfg* cfgs, size_t n,
                            float* grads, size_t cap, double* loss)
{
    if (!ctx || !keys || !cfgs || !grads) return CHAI_ERR_INVALID;
    std::vector<float> x, y, g;
    samples(keys, cfgs, n, x, &y);
    int st = ctx->tuner->mlp()->gradients(x, y, g, loss);
    if (st) return st;
    if (cap < g.size()) return set_error(ctx, CHAI_ERR_INVALID, "mlp gradients: buffer too small");
    std::copy(g.begin(), g.end(), grads);
    return CHAI_OK;
}

int chai_cuda_mlp_weights(chai_cuda_ctx* ctx, float* buf, size_t cap, size_t* count, int set)
{
    if (!ctx) return CHAI_ERR_INVALID;
    return ctx->tuner->mlp()->weights(buf, cap, count, set);
}

}  // extern "C"
