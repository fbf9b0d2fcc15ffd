// Hand-written template pieces of the fused trace kernel ("ID space" kernel,
// the B200 counterpart of enqueue/EnqueueIdSpace.cpp:19-359).  The trace
// translator (trace.cpp) emits one __global__ function per kernel group whose
// body is built from these pieces:
//   - a grid-stride loop in which each thread owns a chunk of 4 consecutive
//     elements of one slot (128-bit ld.global.v4 / st.global.v4 for 32-bit
//     arrays, two 128-bit accesses for f64), grid.y = slot;
//   - register-resident Random123 calls (chai_rng.cuh), one generator call per
//     chunk when the row width is a multiple of the vector length;
//   - per-thread double accumulators for sum / mean / dot_product, reduced by
//     warp shuffles and a shared-memory block tree; each block writes one
//     partial per reduction and slot, and chai_combine_partials (reduce.cu)
//     adds the partials in a fixed order in FP64, so results are
//     deterministic and the final combine is FP64 for any length.
// Embedded verbatim into every runtime-compiled trace kernel.
#pragma once
#ifndef CHAI_TRACE_PRELUDE_CUH
#define CHAI_TRACE_PRELUDE_CUH

namespace chai_k {

typedef unsigned int u32;
typedef long long i64;

template <class T> struct V4 { T v[4]; };

// 4 consecutive elements at p (16-byte aligned for 32-bit types).
template <class T> __device__ __forceinline__ void ld4(const T* __restrict__ p, T (&o)[4])
{
    if constexpr (sizeof(T) == 4) {
        const uint4 r = __ldg(reinterpret_cast<const uint4*>(p));
        o[0] = __builtin_bit_cast(T, r.x); o[1] = __builtin_bit_cast(T, r.y);
        o[2] = __builtin_bit_cast(T, r.z); o[3] = __builtin_bit_cast(T, r.w);
    } else {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        o[0] = (T)a.x; o[1] = (T)a.y; o[2] = (T)b.x; o[3] = (T)b.y;
    }
}

template <class T> __device__ __forceinline__ void st4(T* __restrict__ p, const T (&v)[4])
{
    if constexpr (sizeof(T) == 4) {
        uint4 r;
        r.x = __builtin_bit_cast(unsigned, v[0]); r.y = __builtin_bit_cast(unsigned, v[1]);
        r.z = __builtin_bit_cast(unsigned, v[2]); r.w = __builtin_bit_cast(unsigned, v[3]);
        *reinterpret_cast<uint4*>(p) = r;
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2((double)v[0], (double)v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2((double)v[2], (double)v[3]);
    }
}

// One dot_product term as interp/InterpDotprod.cpp:40-138 forms it: the
// product in the operands' common C type (float * float rounded to f32,
// int * int wrapping in 32 bits, anything * double in f64), widened to
// double for the sum.
template <class A, class B> __device__ __forceinline__ double dot_term(A a, B b) { return (double)(a * b); }
__device__ __forceinline__ double dot_term(int a, int b) { return (double)(int)((unsigned)a * (unsigned)b); }
__device__ __forceinline__ double dot_term(unsigned a, int b) { return (double)(a * (unsigned)b); }
__device__ __forceinline__ double dot_term(int a, unsigned b) { return (double)((unsigned)a * b); }
__device__ __forceinline__ double dot_term(unsigned a, unsigned b) { return (double)(a * b); }

// ld4 / st4 on 4 elements inside a longer per-thread array (rows of a
// multi-row stencil thread)
template <class T> __device__ __forceinline__ void ld4p(const T* __restrict__ p, T* o)
{
    T t[4];
    ld4(p, t);
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2]; o[3] = t[3];
}

template <class T> __device__ __forceinline__ void st4p(T* __restrict__ p, const T* v)
{
    const T t[4] = {v[0], v[1], v[2], v[3]};
    st4(p, t);
}

// 16 bytes of shared memory at p (16-byte aligned) into o[0 .. 16/sizeof(T)).
template <class T> __device__ __forceinline__ void lds_vec(const T* p, T* o)
{
    if constexpr (sizeof(T) == 4) {
        const uint4 r = *reinterpret_cast<const uint4*>(p);
        o[0] = __builtin_bit_cast(T, r.x); o[1] = __builtin_bit_cast(T, r.y);
        o[2] = __builtin_bit_cast(T, r.z); o[3] = __builtin_bit_cast(T, r.w);
    } else {
        const double2 r = *reinterpret_cast<const double2*>(p);
        o[0] = (T)r.x; o[1] = (T)r.y;
    }
}

// Block-wide sum of NRED doubles; thread 0 receives the totals.
template <int NRED, int NT>
__device__ __forceinline__ void block_sum(double (&v)[NRED])
{
    __shared__ double red_smem[NRED][NT / 32];
#pragma unroll
    for (int r = 0; r < NRED; r++) {
        double x = v[r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) red_smem[r][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int r = 0; r < NRED; r++) {
            double x = threadIdx.x < NT / 32 ? red_smem[r][threadIdx.x] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            v[r] = x;
        }
    }
}

// --------------------------------------------------------- stencil tiles
// Tensor map passed by value to a stencil kernel (layout of CUtensorMap).
struct __align__(64) Tmap { unsigned long long opaque[16]; };

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 3-D tiled TMA load (x = innermost, 16-byte aligned) into shared memory
__device__ __forceinline__ void tma_load_3d(void* dst, const Tmap* map, unsigned long long* bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
                 ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

// Bounded wait for phase `parity`: gives up after 2 s, sets *status and
// returns false (the tile is then skipped; nothing waits forever).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int* status)
{
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (;;) {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
                     : "memory");
        if (ok) return true;
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 2000000000ull) {
            atomicExch(status, 201);
            return false;
        }
    }
}

__device__ __forceinline__ long long wrapi(long long v, long long n)
{
    v %= n;
    return v < 0 ? v + n : v;
}

// wrapi for the coordinates a stencil tile reaches (at most one period
// outside [0, n)) without a division; farther values (images narrower than
// a tile and its halo) take the general path
__device__ __forceinline__ long long wrapn(long long v, long long n)
{
    if (v < 0) v += n;
    else if (v >= n) v -= n;
    return (v >= 0 && v < n) ? v : wrapi(v, n);
}

}  // namespace chai_k

#endif
