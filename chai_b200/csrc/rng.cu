// Standalone chai random array fill: the direct-kernel form of the RNG
// statements the trace kernels inline (rng_uniform_make / rng_normal_make,
// api/RngFun.cpp:15-90).  One generator call per vector of 4 (32-bit) or 2
// (f64) elements, 128-bit stores.
#include <cuda_runtime.h>

#include "chai_rng.cuh"
#include "internal.h"

namespace chai {

using namespace chai_rng;

template <int VARIANT, int LAYOUT>
__global__ void __launch_bounds__(256) rng_fill32(void* __restrict__ out, unsigned long long nvec, unsigned seed, int prec,
                                                  int dist, float two_pi, int limits, float len, float lo)
{
    for (unsigned long long v = blockIdx.x * 256ull + threadIdx.x; v < nvec; v += (unsigned long long)gridDim.x * 256) {
        const u32x4 r = raw32<VARIANT, LAYOUT>((unsigned)v, seed, true);
        uint4 o;
        if (prec == CHAI_F32) {
            float f[4];
            if (dist) {
                box_muller_f32(u01_f32(r.x), u01_f32(r.y), two_pi, f[0], f[1]);
                box_muller_f32(u01_f32(r.z), u01_f32(r.w), two_pi, f[2], f[3]);
            } else {
                f[0] = u01_f32(r.x); f[1] = u01_f32(r.y); f[2] = u01_f32(r.z); f[3] = u01_f32(r.w);
                if (limits)
                    for (int j = 0; j < 4; j++) {
                        float t = __fmul_rn(f[j], len);
                        if (lo != 0.0f) t = __fadd_rn(t, lo);
                        f[j] = t;
                    }
            }
            o = make_uint4(__float_as_uint(f[0]), __float_as_uint(f[1]), __float_as_uint(f[2]), __float_as_uint(f[3]));
        } else {
            o = make_uint4(r.x, r.y, r.z, r.w);
        }
        reinterpret_cast<uint4*>(out)[v] = o;
    }
}

template <int VARIANT, int LAYOUT>
__global__ void __launch_bounds__(256) rng_fill64(double* __restrict__ out, unsigned long long nvec,
                                                  unsigned long long seed, int dist, double two_pi, int limits,
                                                  double len, double lo)
{
    for (unsigned long long v = blockIdx.x * 256ull + threadIdx.x; v < nvec; v += (unsigned long long)gridDim.x * 256) {
        const u64x2 r = raw64<VARIANT, LAYOUT>(v, seed);
        double a, b;
        if (dist) {
            box_muller_f64(u01_f64(r.x), u01_f64(r.y), two_pi, a, b);
        } else {
            a = u01_f64(r.x);
            b = u01_f64(r.y);
            if (limits) {
                a = __dmul_rn(a, len); b = __dmul_rn(b, len);
                if (lo != 0.0) { a = __dadd_rn(a, lo); b = __dadd_rn(b, lo); }
            }
        }
        reinterpret_cast<double2*>(out)[v] = make_double2(a, b);
    }
}

int launch_rng_fill(chai_cuda_ctx* ctx, const chai_rng_desc* d, void* out)
{
    const unsigned long long n = (unsigned long long)d->width * d->height * (d->slots ? d->slots : 1);
    if (d->variant != CHAI_RNG_PHILOX && d->variant != CHAI_RNG_THREEFRY)
        return set_error(ctx, CHAI_ERR_INVALID, "rng variant");
    const bool f64 = d->prec == CHAI_F64;
    const unsigned vl = f64 ? 2 : 4;
    if ((d->vec_len && d->vec_len != vl) || (d->width % vl) != 0)
        return set_error(ctx, CHAI_ERR_UNSUPPORTED, "rng_fill: width must be a multiple of the vector length "
                                                    "(use a trace for ragged widths)");
    if ((reinterpret_cast<uintptr_t>(out) & 15) != 0) return set_error(ctx, CHAI_ERR_INVALID, "rng_fill: alignment");
    const unsigned long long nvec = n / vl;
    if (nvec == 0) return CHAI_OK;
    unsigned blocks = (unsigned)std::min<unsigned long long>((nvec + 255) / 256, (unsigned long long)ctx->sm_count * 16);
    const int layout = ctx->cfg.rng_layout;
    const double two_pi = 2.0 * ctx->cfg.rng_pi;
    const double len = d->max_limit - d->min_limit;
    if (f64) {
#define L64(V, LY) rng_fill64<V, LY><<<blocks, 256, 0, ctx->stream>>>((double*)out, nvec, d->seed, (int)d->dist, two_pi, \
                                                                      (int)d->has_limits, len, d->min_limit)
        if (d->variant == CHAI_RNG_PHILOX) { if (layout) L64(1230, 1); else L64(1230, 0); }
        else { if (layout) L64(1231, 1); else L64(1231, 0); }
#undef L64
    } else {
#define L32(V, LY) rng_fill32<V, LY><<<blocks, 256, 0, ctx->stream>>>(out, nvec, (unsigned)d->seed, (int)d->prec, \
                                                                      (int)d->dist, (float)two_pi, (int)d->has_limits, \
                                                                      (float)len, (float)d->min_limit)
        if (d->variant == CHAI_RNG_PHILOX) { if (layout) L32(1230, 1); else L32(1230, 0); }
        else { if (layout) L32(1231, 1); else L32(1231, 0); }
#undef L32
    }
    CHAI_CUDA_TRY(ctx, cudaGetLastError());
    return CHAI_OK;
}

}  // namespace chai
