// Register-resident Random123 generators in chai's layout, for sm_100a.
//
// Follows the OpenCL the reference JIT prints (Random123/R123Philox.cpp:34-523,
// Random123/R123Threefry.cpp:40-535) and the call sites that pick the
// generator and its arguments (kernel/Function.cpp:388-503,
// enqueue/EnqueueAST.cpp:496-545):
//   - 32-bit precisions use Philox4x32-10 / Threefry4x32-20 for vector
//     length 4 and the 2x32 generators for vector lengths 1 and 2; f64 uses
//     Philox2x64-10 / Threefry2x64-20;
//   - key = {vector index, 0xdecafbad[, 0xfacebead, 0x12345678]} and
//     counter = {seed, 0xf00dcafe[, 0xdeadbeef, 0xbeeff00d]} (chai layout),
//     or key word 0 = seed and counter word 0 = vector index (counter layout);
//   - the JIT's Threefry4x32 mixes the fixed lane pairs (0,1),(2,3) in every
//     round (R123Threefry.cpp:230-283), unlike upstream Random123;
//   - uniform = int * 2^-32 + 0.5 (closed interval [0,1]: both 0 and 1 occur),
//     64-bit: int64 * 2^-64 + 0.5;
//   - normal = Box-Muller on lane pairs with the reference's pi constant.
// This header is compiled into the static kernels and embedded verbatim into
// every runtime-compiled trace kernel.
#pragma once
#ifndef CHAI_RNG_CUH
#define CHAI_RNG_CUH

namespace chai_rng {

struct u32x4 { unsigned x, y, z, w; };
struct u64x2 { unsigned long long x, y; };

__device__ __forceinline__ u32x4 philox4x32(unsigned c0, unsigned c1, unsigned c2, unsigned c3,
                                            unsigned k0, unsigned k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const unsigned lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const unsigned lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const unsigned n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return u32x4{c0, c1, c2, c3};
}

__device__ __forceinline__ void philox2x32(unsigned& c0, unsigned& c1, unsigned k)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) k += 0x9E3779B9u;
        const unsigned lo = 0xd256d193u * c0, hi = __umulhi(0xd256d193u, c0);
        c0 = hi ^ k ^ c1;
        c1 = lo;
    }
}

__device__ __forceinline__ u64x2 philox2x64(unsigned long long c0, unsigned long long c1,
                                            unsigned long long k)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) k += 0x9E3779B97F4A7C15ull;
        const unsigned long long lo = 0xD2B74407B1CE6E93ull * c0;
        const unsigned long long hi = __umul64hi(0xD2B74407B1CE6E93ull, c0);
        c0 = hi ^ k ^ c1;
        c1 = lo;
    }
    return u64x2{c0, c1};
}

__device__ __forceinline__ unsigned rotl32(unsigned x, unsigned n) { return __funnelshift_l(x, x, n); }
__device__ __forceinline__ unsigned long long rotl64(unsigned long long x, unsigned n)
{
    return (x << (n & 63)) | (x >> ((64 - n) & 63));
}

// The reference JIT's Threefry4x32-20 (fixed lane pairing).
__device__ __forceinline__ u32x4 threefry4x32(unsigned x0, unsigned x1, unsigned x2, unsigned x3,
                                              unsigned k0, unsigned k1, unsigned k2, unsigned k3)
{
    const unsigned ks[5] = {k0, k1, k2, k3, 0x1BD11BDAu ^ k0 ^ k1 ^ k2 ^ k3};
    const unsigned R0[8] = {10, 11, 13, 23, 6, 17, 25, 18};
    const unsigned R1[8] = {26, 21, 27, 5, 20, 11, 10, 20};
    x0 += ks[0]; x1 += ks[1]; x2 += ks[2]; x3 += ks[3];
#pragma unroll
    for (int r = 0; r < 20; r++) {
        x0 += x1; x1 = rotl32(x1, R0[r % 8]); x1 ^= x0;
        x2 += x3; x3 = rotl32(x3, R1[r % 8]); x3 ^= x2;
        if (r % 4 == 3) {
            const int s = r / 4 + 1;
            x0 += ks[s % 5]; x1 += ks[(s + 1) % 5]; x2 += ks[(s + 2) % 5]; x3 += ks[(s + 3) % 5];
            x3 += (unsigned)s;
        }
    }
    return u32x4{x0, x1, x2, x3};
}

__device__ __forceinline__ void threefry2x32(unsigned& x0, unsigned& x1, unsigned k0, unsigned k1)
{
    const unsigned ks[3] = {k0, k1, 0x1BD11BDAu ^ k0 ^ k1};
    const unsigned R[8] = {13, 15, 26, 6, 17, 29, 16, 24};
    x0 += ks[0]; x1 += ks[1];
#pragma unroll
    for (int r = 0; r < 20; r++) {
        x0 += x1; x1 = rotl32(x1, R[r % 8]); x1 ^= x0;
        if (r % 4 == 3) {
            const int s = r / 4 + 1;
            x0 += ks[s % 3]; x1 += ks[(s + 1) % 3]; x1 += (unsigned)s;
        }
    }
}

__device__ __forceinline__ u64x2 threefry2x64(unsigned long long x0, unsigned long long x1,
                                              unsigned long long k0, unsigned long long k1)
{
    const unsigned long long ks[3] = {k0, k1, 0x1BD11BDAA9FC1A22ull ^ k0 ^ k1};
    const unsigned R[8] = {16, 42, 12, 31, 16, 32, 24, 21};
    x0 += ks[0]; x1 += ks[1];
#pragma unroll
    for (int r = 0; r < 20; r++) {
        x0 += x1; x1 = rotl64(x1, R[r % 8]); x1 ^= x0;
        if (r % 4 == 3) {
            const int s = r / 4 + 1;
            x0 += ks[s % 3]; x1 += ks[(s + 1) % 3]; x1 += (unsigned long long)s;
        }
    }
    return u64x2{x0, x1};
}

// Raw 32-bit lanes of one generator call for vector index `tid`.
// vl4 != 0: 4-lane generator; otherwise the 2-lane one (lanes z, w unused).
template <int VARIANT, int LAYOUT>
__device__ __forceinline__ u32x4 raw32(unsigned tid, unsigned seed, bool vl4)
{
    const unsigned a = LAYOUT ? seed : tid;   // key word 0
    const unsigned b = LAYOUT ? tid : seed;   // counter word 0
    if (vl4) {
        if (VARIANT == 1231)
            return threefry4x32(b, 0xf00dcafeu, 0xdeadbeefu, 0xbeeff00du, a, 0xdecafbadu, 0xfacebeadu,
                                0x12345678u);
        return philox4x32(b, 0xf00dcafeu, 0xdeadbeefu, 0xbeeff00du, a, 0xdecafbadu);
    }
    unsigned c0 = b, c1 = 0xf00dcafeu;
    if (VARIANT == 1231) threefry2x32(c0, c1, a, 0xdecafbadu);
    else philox2x32(c0, c1, a);   // the 2x32 key has one word: {tid}
    return u32x4{c0, c1, 0u, 0u};
}

template <int VARIANT, int LAYOUT>
__device__ __forceinline__ u64x2 raw64(unsigned long long tid, unsigned long long seed)
{
    const unsigned long long a = LAYOUT ? seed : tid;
    const unsigned long long b = LAYOUT ? tid : seed;
    if (VARIANT == 1231) return threefry2x64(b, 0xf00dcafeull, a, 0xdecafbadull);
    return philox2x64(b, 0xf00dcafeull, a);
}

// int * 2^-32 + 0.5 (R123Philox.cpp:405-427); the scaling is exact, so the
// result does not depend on multiply-add contraction.
__device__ __forceinline__ float u01_f32(unsigned r)
{
    return __fadd_rn(__fmul_rn(__int2float_rn((int)r), 2.3283064365386963e-10f), 0.5f);
}
__device__ __forceinline__ double u01_f64(unsigned long long r)
{
    return __dadd_rn(__dmul_rn(__ll2double_rn((long long)r), 5.421010862427522170037E-20), 0.5);
}

// Box-Muller pair (R123Philox.cpp:466-515): z0 = r sin(2 pi u1), z1 = r cos(2 pi u1)
__device__ __forceinline__ void box_muller_f32(float u0, float u1, float two_pi, float& z0, float& z1)
{
    const float r = sqrtf(-2.0f * logf(u0));
    float s, c;
    sincosf(two_pi * u1, &s, &c);
    z0 = r * s;
    z1 = r * c;
}
__device__ __forceinline__ void box_muller_f64(double u0, double u1, double two_pi, double& z0, double& z1)
{
    const double r = sqrt(-2.0 * log(u0));
    double s, c;
    sincos(two_pi * u1, &s, &c);
    z0 = r * s;
    z1 = r * c;
}

}  // namespace chai_rng

#endif
