// Inline OpenCL kernels (ProgramCL): OpenCL C text -> CUDA for NVRTC, and the
// translator step that launches one.
//
// Reference: api/ProgramCL.cpp (argument kinds from the kernel signature:
// __global / image2d_t arrays, __local memory, scalars), jitast/AstOpenCL.cpp
// (the program text travels with the trace), enqueue/EnqueueOpenCL.cpp (the
// kernel is enqueued with the arrays' device buffers, the __local sizes and
// the scalars as arguments, over the NDRange the caller gave).
//
// The OpenCL C is compiled, not interpreted: a prelude maps the work-item
// functions (get_global_id ... get_num_groups), barrier / mem_fence and the
// usual type names onto CUDA; the address-space qualifiers are rewritten token
// by token (__kernel -> extern "C" __global__, __global / __private removed,
// __constant -> const, __local -> __shared__ in bodies).  A __local pointer
// parameter becomes a plain pointer that the kernel body points into its
// dynamic shared memory at the offset its size gives.
//
// OpenCL C 1.2 beyond the scalar language (the built-ins of its section 6.12):
// vector types (charN ... doubleN, N = 2, 3, 4, 8, 16) as chai_cl::vec with
// the component-wise operators, vector literals, swizzles (.xy, .s01,
// .lo / .hi / .even / .odd, as values or assigned to), convert_* with _sat
// and the four rounding modes, as_*, vloadN / vstoreN, the math, integer,
// common, geometric and relational built-ins on vectors, atomic_* / atom_*,
// async_work_group_copy; and image2d_t parameters: the array's storage read
// and written as rows of 16-byte RGBA texels (read_imagef / read_imagei /
// read_imageui with nearest or bilinear samplers and the five addressing
// modes, write_image*), the layout the reference's OpenCL images give an
// array (vendor/OCLdevice.cpp:251-285: RGBA, 32-bit channels, an f64 array
// as two values per texel).
#include <cuda_runtime.h>

#include <cctype>
#include <cstdint>
#include <cstring>
#include <sstream>

#include "internal.h"
#include "jit.h"
#include "trace.h"

namespace chai {

static const char* kOpenCLPrelude = R"cl(
// ---- OpenCL C on sm_100a (inline ProgramCL kernels)
typedef unsigned int uint;
typedef unsigned long long ulong;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef decltype(sizeof(0)) size_t;
typedef int event_t;
typedef unsigned int sampler_t;
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
// sampler fields: coordinates (bit 0), addressing (bits 1-3), filter (bit 4)
#define CLK_NORMALIZED_COORDS_FALSE 0u
#define CLK_NORMALIZED_COORDS_TRUE 1u
#define CLK_ADDRESS_NONE 0u
#define CLK_ADDRESS_CLAMP_TO_EDGE 2u
#define CLK_ADDRESS_CLAMP 4u
#define CLK_ADDRESS_REPEAT 6u
#define CLK_ADDRESS_MIRRORED_REPEAT 8u
#define CLK_FILTER_NEAREST 0u
#define CLK_FILTER_LINEAR 16u
__device__ __forceinline__ size_t get_global_id(uint d)
{ return d == 0 ? (size_t)blockIdx.x * blockDim.x + threadIdx.x
       : d == 1 ? (size_t)blockIdx.y * blockDim.y + threadIdx.y : (size_t)blockIdx.z * blockDim.z + threadIdx.z; }
__device__ __forceinline__ size_t get_local_id(uint d) { return d == 0 ? threadIdx.x : d == 1 ? threadIdx.y : threadIdx.z; }
__device__ __forceinline__ size_t get_group_id(uint d) { return d == 0 ? blockIdx.x : d == 1 ? blockIdx.y : blockIdx.z; }
__device__ __forceinline__ size_t get_local_size(uint d) { return d == 0 ? blockDim.x : d == 1 ? blockDim.y : blockDim.z; }
__device__ __forceinline__ size_t get_num_groups(uint d) { return d == 0 ? gridDim.x : d == 1 ? gridDim.y : gridDim.z; }
__device__ __forceinline__ size_t get_global_size(uint d) { return get_num_groups(d) * get_local_size(d); }
__device__ __forceinline__ size_t get_global_offset(uint) { return 0; }
__device__ __forceinline__ uint get_work_dim() { return CHAI_CL_WORK_DIM; }
__device__ __forceinline__ void barrier(int) { __syncthreads(); }
__device__ __forceinline__ void mem_fence(int) { __threadfence_block(); }
__device__ __forceinline__ void read_mem_fence(int) { __threadfence_block(); }
__device__ __forceinline__ void write_mem_fence(int) { __threadfence_block(); }
namespace chai_cl {
template <bool B, class R = void> struct en_if {};
template <class R> struct en_if<true, R> { typedef R type; };
template <class A, class B> struct same { static constexpr bool value = false; };
template <class A> struct same<A, A> { static constexpr bool value = true; };
template <class T> struct id { typedef T type; };
template <class T> struct num { static constexpr bool value = false, fp = false, sgn = false; };
#define CHAI_CL_NUM(T, F, S) template <> struct num<T> { static constexpr bool value = true, fp = F, sgn = S; };
CHAI_CL_NUM(bool, false, false) CHAI_CL_NUM(char, false, true) CHAI_CL_NUM(signed char, false, true)
CHAI_CL_NUM(unsigned char, false, false) CHAI_CL_NUM(short, false, true) CHAI_CL_NUM(unsigned short, false, false)
CHAI_CL_NUM(int, false, true) CHAI_CL_NUM(unsigned int, false, false) CHAI_CL_NUM(long, false, true)
CHAI_CL_NUM(unsigned long, false, false) CHAI_CL_NUM(long long, false, true)
CHAI_CL_NUM(unsigned long long, false, false) CHAI_CL_NUM(float, true, true) CHAI_CL_NUM(double, true, true)
#undef CHAI_CL_NUM
template <class S, class R> using if_num = typename en_if<num<S>::value, R>::type;
template <class S, class R> using if_int = typename en_if<num<S>::value && !num<S>::fp, R>::type;
template <class S, class R> using if_fp = typename en_if<num<S>::fp, R>::type;
template <int B> struct uint_of;
template <> struct uint_of<1> { typedef unsigned char type; };
template <> struct uint_of<2> { typedef unsigned short type; };
template <> struct uint_of<4> { typedef unsigned int type; };
template <> struct uint_of<8> { typedef unsigned long long type; };
template <class T> using utype = typename uint_of<sizeof(T)>::type;
template <class T> __device__ __forceinline__ bool msb(T x) { return (((utype<T>)x) >> (8 * sizeof(T) - 1)) != 0; }
template <class D> __device__ __forceinline__ constexpr D maxv()
{ return num<D>::sgn ? (D)(((utype<D>)~(utype<D>)0) >> 1) : (D)~(utype<D>)0; }
template <class D> __device__ __forceinline__ constexpr D minv()
{ return num<D>::sgn ? (D)((utype<D>)1 << (8 * sizeof(D) - 1)) : D(0); }
// reinterpretation of the bits of one object as another of the same size
template <class D, class S> __device__ __forceinline__ D as_type(const S& s)
{
    static_assert(sizeof(D) == sizeof(S), "as_type: operand and result sizes differ");
    D d;
    memcpy(&d, &s, sizeof(D));
    return d;
}
}  // namespace chai_cl
// ---- scalar built-ins
template <class T> __device__ __forceinline__ chai_cl::if_num<T, T> mad(T a, T b, T c) { return a * b + c; }
template <class T> __device__ __forceinline__ chai_cl::if_num<T, T> clamp(T x, T lo, T hi)
{
    if constexpr (chai_cl::num<T>::fp) return fmin(fmax(x, lo), hi);
    else return x < lo ? lo : (x > hi ? hi : x);
}
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> mix(T x, T y, T a) { return x + (y - x) * a; }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> step(T edge, T x) { return x < edge ? T(0) : T(1); }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> smoothstep(T e0, T e1, T x)
{
    const T t = clamp((x - e0) / (e1 - e0), T(0), T(1));
    return t * t * (T(3) - T(2) * t);
}
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> sign(T x)
{ return x > T(0) ? T(1) : x < T(0) ? T(-1) : x == T(0) ? x : T(0); }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> degrees(T r) { return r * T(57.295779513082320876798154814105); }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> radians(T d) { return d * T(0.017453292519943295769236907684886); }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> dot(T a, T b) { return a * b; }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> length(T a) { return fabs(a); }
template <class T> __device__ __forceinline__ chai_cl::if_fp<T, T> distance(T a, T b) { return fabs(a - b); }
template <class T, class C> __device__ __forceinline__ chai_cl::if_num<T, T> select(T a, T b, C c) { return c ? b : a; }
template <class T> __device__ __forceinline__ chai_cl::if_int<T, int> any(T x) { return chai_cl::msb(x); }
template <class T> __device__ __forceinline__ chai_cl::if_int<T, int> all(T x) { return chai_cl::msb(x); }
template <class T> __device__ __forceinline__ chai_cl::if_num<T, T> bitselect(T a, T b, T c)
{
    typedef chai_cl::utype<T> U;
    const U x = chai_cl::as_type<U>(a), y = chai_cl::as_type<U>(b), m = chai_cl::as_type<U>(c);
    return chai_cl::as_type<T>((U)((x & ~m) | (y & m)));
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> clz(T x)
{
    if constexpr (sizeof(T) == 8) return (T)__clzll((long long)x);
    else return (T)(__clz((int)(unsigned)(chai_cl::utype<T>)x) - 8 * (4 - (int)sizeof(T)));
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> popcount(T x)
{
    if constexpr (sizeof(T) == 8) return (T)__popcll((unsigned long long)x);
    else return (T)__popc((unsigned)(chai_cl::utype<T>)x);
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> rotate(T v, T i)
{
    typedef chai_cl::utype<T> U;
    const int b = 8 * (int)sizeof(T), s = (int)((U)i & (U)(b - 1));
    const U u = (U)v;
    return s ? (T)(U)((u << s) | (u >> (b - s))) : v;
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> mul_hi(T a, T b)
{
    if constexpr (sizeof(T) == 8 && chai_cl::num<T>::sgn) return (T)__mul64hi((long long)a, (long long)b);
    else if constexpr (sizeof(T) == 8) return (T)__umul64hi((unsigned long long)a, (unsigned long long)b);
    else if constexpr (sizeof(T) == 4 && chai_cl::num<T>::sgn) return (T)__mulhi((int)a, (int)b);
    else if constexpr (sizeof(T) == 4) return (T)__umulhi((unsigned)a, (unsigned)b);
    else return (T)(((int)a * (int)b) >> (8 * sizeof(T)));
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> mul24(T a, T b) { return (T)(a * b); }
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> mad24(T a, T b, T c) { return (T)(a * b + c); }
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> hadd(T x, T y) { return (T)((x >> 1) + (y >> 1) + (x & y & 1)); }
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> rhadd(T x, T y) { return (T)((x >> 1) + (y >> 1) + ((x | y) & 1)); }
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> add_sat(T a, T b)
{
    if constexpr (sizeof(T) < 8) {
        const long long r = (long long)a + (long long)b;
        return r < (long long)chai_cl::minv<T>() ? chai_cl::minv<T>() : r > (long long)chai_cl::maxv<T>() ? chai_cl::maxv<T>() : (T)r;
    } else if constexpr (chai_cl::num<T>::sgn) {
        const T r = (T)((unsigned long long)a + (unsigned long long)b);
        return (a > 0 && b > 0 && r < 0) ? chai_cl::maxv<T>() : (a < 0 && b < 0 && r >= 0) ? chai_cl::minv<T>() : r;
    } else {
        const T r = (T)(a + b);
        return r < a ? chai_cl::maxv<T>() : r;
    }
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, T> sub_sat(T a, T b)
{
    if constexpr (sizeof(T) < 8) {
        const long long r = (long long)a - (long long)b;
        return r < (long long)chai_cl::minv<T>() ? chai_cl::minv<T>() : r > (long long)chai_cl::maxv<T>() ? chai_cl::maxv<T>() : (T)r;
    } else if constexpr (chai_cl::num<T>::sgn) {
        const T r = (T)((unsigned long long)a - (unsigned long long)b);
        return (a >= 0 && b < 0 && r < 0) ? chai_cl::maxv<T>() : (a < 0 && b > 0 && r >= 0) ? chai_cl::minv<T>() : r;
    } else {
        return a < b ? T(0) : (T)(a - b);
    }
}
template <class T> __device__ __forceinline__ chai_cl::if_int<T, chai_cl::utype<T>> abs_diff(T a, T b)
{
    typedef chai_cl::utype<T> U;
    return a > b ? (U)((U)a - (U)b) : (U)((U)b - (U)a);
}
__device__ __forceinline__ float fract(float x, float* ip) { const float f = floorf(x); *ip = f; return fminf(x - f, 0x1.fffffep-1f); }
__device__ __forceinline__ double fract(double x, double* ip) { const double f = floor(x); *ip = f; return fmin(x - f, 0x1.fffffffffffffp-1); }
__device__ __forceinline__ float sincos(float x, float* c) { float s; sincosf(x, &s, c); return s; }
__device__ __forceinline__ double sincos(double x, double* c) { double s; sincos(x, &s, c); return s; }
#define native_exp exp
#define native_log log
#define native_sqrt sqrt
#define native_rsqrt rsqrt
#define native_sin sin
#define native_cos cos
#define native_tan tan
#define native_powr pow
#define native_exp2 exp2
#define native_exp10 exp10
#define native_log2 log2
#define native_log10 log10
#define native_divide(a, b) ((a) / (b))
#define native_recip(x) (1 / (x))
#define half_exp exp
#define half_log log
#define half_sqrt sqrt
#define half_rsqrt rsqrt
#define half_sin sin
#define half_cos cos
#define half_divide(a, b) ((a) / (b))
#define half_recip(x) (1 / (x))
#define powr pow
#define fast_length length
#define fast_distance distance
#define fast_normalize normalize
__device__ __forceinline__ double pown(double x, int n) { return pow(x, (double)n); }
__device__ __forceinline__ float pown(float x, int n) { return powf(x, (float)n); }
__device__ __forceinline__ double rootn(double x, int n) { return pow(x, 1.0 / n); }
__device__ __forceinline__ float rootn(float x, int n) { return powf(x, 1.0f / n); }
// ---- atomics on __global / __local words (OpenCL 1.1 atomic_*, and the atom_* names of the 64-bit extensions)
namespace chai_cl {
template <class T> struct wide { static constexpr bool value = sizeof(T) == 8 && !num<T>::fp; };
}
template <class T> __device__ __forceinline__ T atomic_add(volatile T* p, typename chai_cl::id<T>::type v)
{
    if constexpr (chai_cl::wide<T>::value) return (T)atomicAdd((unsigned long long*)p, (unsigned long long)v);
    else return atomicAdd((T*)p, v);
}
template <class T> __device__ __forceinline__ T atomic_sub(volatile T* p, typename chai_cl::id<T>::type v)
{
    if constexpr (chai_cl::wide<T>::value) return (T)atomicAdd((unsigned long long*)p, 0ull - (unsigned long long)v);
    else if constexpr (chai_cl::num<T>::fp) return atomicAdd((T*)p, -v);
    else return atomicSub((T*)p, v);
}
template <class T> __device__ __forceinline__ T atomic_xchg(volatile T* p, typename chai_cl::id<T>::type v)
{
    if constexpr (chai_cl::wide<T>::value) return (T)atomicExch((unsigned long long*)p, (unsigned long long)v);
    else return atomicExch((T*)p, v);
}
template <class T> __device__ __forceinline__ T atomic_inc(volatile T* p) { return atomic_add(p, T(1)); }
template <class T> __device__ __forceinline__ T atomic_dec(volatile T* p) { return atomic_sub(p, T(1)); }
template <class T> __device__ __forceinline__ T atomic_cmpxchg(volatile T* p, typename chai_cl::id<T>::type cmp,
                                                               typename chai_cl::id<T>::type v)
{
    if constexpr (chai_cl::wide<T>::value)
        return (T)atomicCAS((unsigned long long*)p, (unsigned long long)cmp, (unsigned long long)v);
    else return atomicCAS((T*)p, cmp, v);
}
#define CHAI_CL_ATOMIC_MINMAX(name, fn)                                                                  \
template <class T> __device__ __forceinline__ T name(volatile T* p, typename chai_cl::id<T>::type v)      \
{                                                                                                        \
    if constexpr (chai_cl::wide<T>::value && chai_cl::num<T>::sgn) return (T)fn((long long*)p, (long long)v); \
    else if constexpr (chai_cl::wide<T>::value) return (T)fn((unsigned long long*)p, (unsigned long long)v); \
    else return fn((T*)p, v);                                                                            \
}
CHAI_CL_ATOMIC_MINMAX(atomic_min, atomicMin)
CHAI_CL_ATOMIC_MINMAX(atomic_max, atomicMax)
#define CHAI_CL_ATOMIC_BITS(name, fn)                                                                    \
template <class T> __device__ __forceinline__ T name(volatile T* p, typename chai_cl::id<T>::type v)      \
{                                                                                                        \
    if constexpr (chai_cl::wide<T>::value) return (T)fn((unsigned long long*)p, (unsigned long long)v);  \
    else return fn((T*)p, v);                                                                            \
}
CHAI_CL_ATOMIC_BITS(atomic_and, atomicAnd)
CHAI_CL_ATOMIC_BITS(atomic_or, atomicOr)
CHAI_CL_ATOMIC_BITS(atomic_xor, atomicXor)
#define atom_add atomic_add
#define atom_sub atomic_sub
#define atom_xchg atomic_xchg
#define atom_inc atomic_inc
#define atom_dec atomic_dec
#define atom_cmpxchg atomic_cmpxchg
#define atom_min atomic_min
#define atom_max atomic_max
#define atom_and atomic_and
#define atom_or atomic_or
#define atom_xor atomic_xor
// ---- work-group copies (done by the group's work items when issued; the wait is a barrier)
__device__ __forceinline__ size_t chai_cl_local_linear_id()
{ return ((size_t)threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x; }
template <class T> __device__ __forceinline__ event_t async_work_group_copy(T* dst, const T* src, size_t n, event_t e)
{
    const size_t g = (size_t)blockDim.x * blockDim.y * blockDim.z;
    for (size_t i = chai_cl_local_linear_id(); i < n; i += g) dst[i] = src[i];
    return e;
}
template <class T>
__device__ __forceinline__ event_t async_work_group_strided_copy(T* dst, const T* src, size_t n, size_t stride, event_t e)
{
    const size_t g = (size_t)blockDim.x * blockDim.y * blockDim.z;
    const bool to_local = __isShared(dst);
    for (size_t i = chai_cl_local_linear_id(); i < n; i += g) {
        if (to_local) dst[i] = src[i * stride];
        else dst[i * stride] = src[i];
    }
    return e;
}
__device__ __forceinline__ void wait_group_events(int, event_t*) { __syncthreads(); }
template <class T> __device__ __forceinline__ void prefetch(const T*, size_t) {}
)cl";

static const char* kOpenCLVectors = R"cl(
// ---- OpenCL vector types: chai_cl::vec<T, N> (N = 2, 3, 4, 8, 16; a 3-vector
// is laid out and aligned as a 4-vector), component access by .x .y .z .w
// members and, after the text rewrite, by swizzle methods
namespace chai_cl {
template <int... I> struct iseq {};
template <int B, int S, int K, int... I> struct mkseq : mkseq<B, S, K - 1, B + S * (K - 1), I...> {};
template <int B, int S, int... I> struct mkseq<B, S, 0, I...> { typedef iseq<I...> type; };
template <class T, int N> struct vec;
template <class T, int N, int... I> struct swz;
#define CHAI_CL_FOR(N) _Pragma("unroll") for (int i = 0; i < (N); i++)
#define CHAI_CL_VEC_COMMON(N_)                                                                         \
    typedef T elem;                                                                                    \
    static constexpr int n = N_, H = (N_ == 3 ? 4 : N_) / 2;                                           \
    vec() = default;                                                                                   \
    template <int... I> __device__ auto chai_r(iseq<I...>) const                                       \
    {                                                                                                  \
        if constexpr (sizeof...(I) == 1) return T(c(I...));                                            \
        else return vec<T, (int)sizeof...(I)>(c(I)...);                                                \
    }                                                                                                  \
    template <int... I> __device__ decltype(auto) chai_l(iseq<I...>)                                   \
    {                                                                                                  \
        if constexpr (sizeof...(I) == 1) return c(I...);                                               \
        else return swz<T, N_, I...>{this};                                                            \
    }                                                                                                  \
    template <int... I> __device__ auto chai_swr() const { return chai_r(iseq<I...>()); }              \
    template <int... I> __device__ decltype(auto) chai_swl() { return chai_l(iseq<I...>()); }          \
    template <int I> __device__ T& chai_sw1() { return c(I); }                                         \
    template <int I> __device__ T chai_sw1() const { return c(I); }                                    \
    __device__ auto chai_lo() const { return chai_r(typename mkseq<0, 1, H>::type()); }                \
    __device__ auto chai_hi() const { return chai_r(typename mkseq<H, 1, H>::type()); }                \
    __device__ auto chai_even() const { return chai_r(typename mkseq<0, 2, H>::type()); }              \
    __device__ auto chai_odd() const { return chai_r(typename mkseq<1, 2, H>::type()); }               \
    __device__ decltype(auto) chai_lo_l() { return chai_l(typename mkseq<0, 1, H>::type()); }          \
    __device__ decltype(auto) chai_hi_l() { return chai_l(typename mkseq<H, 1, H>::type()); }          \
    __device__ decltype(auto) chai_even_l() { return chai_l(typename mkseq<0, 2, H>::type()); }        \
    __device__ decltype(auto) chai_odd_l() { return chai_l(typename mkseq<1, 2, H>::type()); }
template <class T> struct alignas(2 * sizeof(T)) vec<T, 2> {
    T x, y;
    __device__ constexpr vec(T s) : x(s), y(s) {}
    __device__ constexpr vec(T a0, T a1) : x(a0), y(a1) {}
    __device__ T& c(int i) { return i ? y : x; }
    __device__ constexpr T c(int i) const { return i ? y : x; }
    CHAI_CL_VEC_COMMON(2)
};
template <class T> struct alignas(4 * sizeof(T)) vec<T, 3> {
    T x, y, z, chai_w;
    __device__ constexpr vec(T s) : x(s), y(s), z(s), chai_w(s) {}
    __device__ constexpr vec(T a0, T a1, T a2) : x(a0), y(a1), z(a2), chai_w(T(0)) {}
    __device__ T& c(int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : chai_w; }
    __device__ constexpr T c(int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : chai_w; }
    CHAI_CL_VEC_COMMON(3)
};
template <class T> struct alignas(4 * sizeof(T)) vec<T, 4> {
    T x, y, z, w;
    __device__ constexpr vec(T s) : x(s), y(s), z(s), w(s) {}
    __device__ constexpr vec(T a0, T a1, T a2, T a3) : x(a0), y(a1), z(a2), w(a3) {}
    __device__ T& c(int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
    __device__ constexpr T c(int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
    CHAI_CL_VEC_COMMON(4)
};
template <class T> struct alignas(8 * sizeof(T)) vec<T, 8> {
    T chai_s[8];
    __device__ constexpr vec(T s) : chai_s{s, s, s, s, s, s, s, s} {}
    __device__ constexpr vec(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7)
        : chai_s{a0, a1, a2, a3, a4, a5, a6, a7} {}
    __device__ T& c(int i) { return chai_s[i]; }
    __device__ constexpr T c(int i) const { return chai_s[i]; }
    CHAI_CL_VEC_COMMON(8)
};
template <class T> struct alignas(16 * sizeof(T)) vec<T, 16> {
    T chai_s[16];
    __device__ constexpr vec(T s) : chai_s{s, s, s, s, s, s, s, s, s, s, s, s, s, s, s, s} {}
    __device__ constexpr vec(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7, T a8, T a9, T a10, T a11, T a12,
                             T a13, T a14, T a15)
        : chai_s{a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15} {}
    __device__ T& c(int i) { return chai_s[i]; }
    __device__ constexpr T c(int i) const { return chai_s[i]; }
    CHAI_CL_VEC_COMMON(16)
};
// a swizzle written to: v.xy = ..., v.lo += ...
template <class T, int N, int... I> struct swz {
    vec<T, N>* p;
    typedef vec<T, (int)sizeof...(I)> V;
    __device__ operator V() const { return V(p->c(I)...); }
    __device__ swz& operator=(const V& v)
    {
        int k = 0;
        ((p->c(I) = v.c(k++)), ...);
        return *this;
    }
    __device__ swz& operator=(const swz& o) { return *this = V(o); }
    template <class S> __device__ if_num<S, swz&> operator=(S s) { return *this = V((T)s); }
    __device__ swz& operator++() { return *this = V(*this) + T(1); }
    __device__ swz& operator--() { return *this = V(*this) - T(1); }
    __device__ V operator++(int) { const V o = *this; *this = o + T(1); return o; }
    __device__ V operator--(int) { const V o = *this; *this = o - T(1); return o; }
#define CHAI_CL_SWZ_OP(op) template <class R> __device__ swz& operator op##=(const R& r) { return *this = V(*this) op r; }
    CHAI_CL_SWZ_OP(+) CHAI_CL_SWZ_OP(-) CHAI_CL_SWZ_OP(*) CHAI_CL_SWZ_OP(/) CHAI_CL_SWZ_OP(%)
    CHAI_CL_SWZ_OP(&) CHAI_CL_SWZ_OP(|) CHAI_CL_SWZ_OP(^) CHAI_CL_SWZ_OP(<<) CHAI_CL_SWZ_OP(>>)
#undef CHAI_CL_SWZ_OP
};
// the integer vector a comparison yields: -1 (all bits) where true, 0 where false
template <class T> struct cmp_t { typedef int type; };
template <> struct cmp_t<double> { typedef long long type; };
template <> struct cmp_t<long> { typedef long long type; };
template <> struct cmp_t<unsigned long> { typedef long long type; };
template <> struct cmp_t<long long> { typedef long long type; };
template <> struct cmp_t<unsigned long long> { typedef long long type; };
template <> struct cmp_t<char> { typedef signed char type; };
template <> struct cmp_t<signed char> { typedef signed char type; };
template <> struct cmp_t<unsigned char> { typedef signed char type; };
template <> struct cmp_t<short> { typedef short type; };
template <> struct cmp_t<unsigned short> { typedef short type; };
template <class T, int N> using cvec = vec<typename cmp_t<T>::type, N>;
#define CHAI_CL_ARITH(op)                                                                              \
template <class T, int N> __device__ vec<T, N> operator op(const vec<T, N>& a, const vec<T, N>& b)      \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = (T)(a.c(i) op b.c(i)); return r; }                                \
template <class T, int N, class S> __device__ if_num<S, vec<T, N>> operator op(const vec<T, N>& a, S b)  \
{ return a op vec<T, N>((T)b); }                                                                         \
template <class T, int N, class S> __device__ if_num<S, vec<T, N>> operator op(S a, const vec<T, N>& b)  \
{ return vec<T, N>((T)a) op b; }                                                                         \
template <class T, int N, class R> __device__ vec<T, N>& operator op##=(vec<T, N>& a, const R& b) { return a = a op b; }
CHAI_CL_ARITH(+) CHAI_CL_ARITH(-) CHAI_CL_ARITH(*) CHAI_CL_ARITH(/) CHAI_CL_ARITH(%)
CHAI_CL_ARITH(&) CHAI_CL_ARITH(|) CHAI_CL_ARITH(^)
#undef CHAI_CL_ARITH
// shifts take the count modulo the component width
#define CHAI_CL_SHIFT(op)                                                                              \
template <class T, int N, class U> __device__ vec<T, N> operator op(const vec<T, N>& a, const vec<U, N>& b) \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = (T)(a.c(i) op (int)(b.c(i) & (U)(8 * sizeof(T) - 1))); return r; } \
template <class T, int N, class S> __device__ if_num<S, vec<T, N>> operator op(const vec<T, N>& a, S b)  \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = (T)(a.c(i) op (int)(b & (S)(8 * sizeof(T) - 1))); return r; }     \
template <class T, int N, class R> __device__ vec<T, N>& operator op##=(vec<T, N>& a, const R& b) { return a = a op b; }
CHAI_CL_SHIFT(<<) CHAI_CL_SHIFT(>>)
#undef CHAI_CL_SHIFT
template <class T, int N> __device__ vec<T, N> operator-(const vec<T, N>& a)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = (T)-a.c(i); return r; }
template <class T, int N> __device__ vec<T, N> operator+(const vec<T, N>& a) { return a; }
template <class T, int N> __device__ vec<T, N> operator~(const vec<T, N>& a)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = (T)~a.c(i); return r; }
template <class T, int N> __device__ cvec<T, N> operator!(const vec<T, N>& a)
{ cvec<T, N> r; CHAI_CL_FOR(N) r.c(i) = a.c(i) ? 0 : -1; return r; }
template <class T, int N> __device__ vec<T, N>& operator++(vec<T, N>& a) { return a = a + T(1); }
template <class T, int N> __device__ vec<T, N>& operator--(vec<T, N>& a) { return a = a - T(1); }
template <class T, int N> __device__ vec<T, N> operator++(vec<T, N>& a, int) { const vec<T, N> o = a; a = o + T(1); return o; }
template <class T, int N> __device__ vec<T, N> operator--(vec<T, N>& a, int) { const vec<T, N> o = a; a = o - T(1); return o; }
#define CHAI_CL_CMP(op)                                                                                \
template <class T, int N> __device__ cvec<T, N> operator op(const vec<T, N>& a, const vec<T, N>& b)      \
{ cvec<T, N> r; CHAI_CL_FOR(N) r.c(i) = (a.c(i) op b.c(i)) ? -1 : 0; return r; }                         \
template <class T, int N, class S> __device__ if_num<S, cvec<T, N>> operator op(const vec<T, N>& a, S b) \
{ return a op vec<T, N>((T)b); }                                                                         \
template <class T, int N, class S> __device__ if_num<S, cvec<T, N>> operator op(S a, const vec<T, N>& b) \
{ return vec<T, N>((T)a) op b; }
CHAI_CL_CMP(==) CHAI_CL_CMP(!=) CHAI_CL_CMP(<) CHAI_CL_CMP(>) CHAI_CL_CMP(<=) CHAI_CL_CMP(>=)
CHAI_CL_CMP(&&) CHAI_CL_CMP(||)
#undef CHAI_CL_CMP
// vector literals: (float4)(a, b, c, d), (float4)(v2, a, b), (float4)(s)
template <class V> struct ncomp { static constexpr int n = 1; };
template <class T, int N> struct ncomp<vec<T, N>> { static constexpr int n = N; };
template <class T, class S> __device__ __forceinline__ if_num<S, void> put(T* o, int& k, const S& s) { o[k++] = (T)s; }
template <class T, class U, int M> __device__ __forceinline__ void put(T* o, int& k, const vec<U, M>& v)
{ CHAI_CL_FOR(M) o[k++] = (T)v.c(i); }
template <class V, class... A> __device__ __forceinline__ V make(const A&... a)
{
    typedef typename V::elem T;
    constexpr int total = (0 + ... + ncomp<A>::n);
    static_assert(total == V::n || (sizeof...(A) == 1 && total == 1), "vector literal: wrong number of components");
    if constexpr (sizeof...(A) == 1 && total == 1) {
        return V((T)(a, ...));
    } else {
        T t[V::n];
        int k = 0;
        (put(t, k, a), ...);
        V r;
        CHAI_CL_FOR(V::n) r.c(i) = t[i];
        return r;
    }
}
// convert_<type>[N][_sat][_rte|_rtz|_rtp|_rtn]: M = 0 default, 1 rte, 2 rtz, 3 rtp, 4 rtn
template <class D, int SAT, int M, class S> __device__ __forceinline__ D cvt1(S x)
{
    if constexpr (num<D>::fp && !num<S>::fp) {
        if constexpr (sizeof(S) <= 2 || (same<D, double>::value && sizeof(S) == 4)) return (D)x;
        else if constexpr (same<D, float>::value && sizeof(S) == 4 && num<S>::sgn)
            return M == 2 ? __int2float_rz((int)x) : M == 3 ? __int2float_ru((int)x) : M == 4 ? __int2float_rd((int)x)
                                                                                             : __int2float_rn((int)x);
        else if constexpr (same<D, float>::value && sizeof(S) == 4)
            return M == 2 ? __uint2float_rz((unsigned)x) : M == 3 ? __uint2float_ru((unsigned)x)
                 : M == 4 ? __uint2float_rd((unsigned)x) : __uint2float_rn((unsigned)x);
        else if constexpr (same<D, float>::value && num<S>::sgn)
            return M == 2 ? __ll2float_rz((long long)x) : M == 3 ? __ll2float_ru((long long)x)
                 : M == 4 ? __ll2float_rd((long long)x) : __ll2float_rn((long long)x);
        else if constexpr (same<D, float>::value)
            return M == 2 ? __ull2float_rz((unsigned long long)x) : M == 3 ? __ull2float_ru((unsigned long long)x)
                 : M == 4 ? __ull2float_rd((unsigned long long)x) : __ull2float_rn((unsigned long long)x);
        else if constexpr (num<S>::sgn)
            return M == 2 ? __ll2double_rz((long long)x) : M == 3 ? __ll2double_ru((long long)x)
                 : M == 4 ? __ll2double_rd((long long)x) : __ll2double_rn((long long)x);
        else
            return M == 2 ? __ull2double_rz((unsigned long long)x) : M == 3 ? __ull2double_ru((unsigned long long)x)
                 : M == 4 ? __ull2double_rd((unsigned long long)x) : __ull2double_rn((unsigned long long)x);
    } else if constexpr (same<D, float>::value && same<S, double>::value) {
        return M == 2 ? __double2float_rz(x) : M == 3 ? __double2float_ru(x) : M == 4 ? __double2float_rd(x)
                                                                                     : __double2float_rn(x);
    } else if constexpr (num<D>::fp) {
        return (D)x;
    } else if constexpr (num<S>::fp) {
        double y = (double)x;
        y = M == 1 ? ::rint(y) : M == 3 ? ::ceil(y) : M == 4 ? ::floor(y) : ::trunc(y);
        if constexpr (SAT != 0) {
            if (y != y) return D(0);
            if (y < (double)minv<D>()) return minv<D>();
            if (y >= (double)maxv<D>()) return maxv<D>();
        }
        return (D)y;
    } else {
        if constexpr (SAT != 0 && num<S>::sgn) {
            const long long v = (long long)x;
            if (v < (long long)minv<D>()) return minv<D>();
            if (v > 0 && (unsigned long long)v > (unsigned long long)maxv<D>()) return maxv<D>();
        } else if constexpr (SAT != 0) {
            if ((unsigned long long)x > (unsigned long long)maxv<D>()) return maxv<D>();
        }
        return (D)x;
    }
}
template <class D, int N, int SAT, int M, class S> __device__ __forceinline__ if_num<S, D> convert(S x)
{ return cvt1<D, SAT, M>(x); }
template <class D, int N, int SAT, int M, class S> __device__ __forceinline__ vec<D, N> convert(const vec<S, N>& v)
{ vec<D, N> r; CHAI_CL_FOR(N) r.c(i) = cvt1<D, SAT, M>(v.c(i)); return r; }
// built-ins on vectors: the scalar function on each component
#define CHAI_CL_LIFT1(f)                                                                               \
template <class T, int N> __device__ __forceinline__ auto f(const vec<T, N>& a)                          \
{ vec<decltype(::f(a.c(0))), N> r; CHAI_CL_FOR(N) r.c(i) = ::f(a.c(i)); return r; }
#define CHAI_CL_LIFT2(f)                                                                               \
template <class T, int N> __device__ __forceinline__ vec<T, N> f(const vec<T, N>& a, const vec<T, N>& b)  \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::f(a.c(i), b.c(i)); return r; }                                  \
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> f(const vec<T, N>& a, S b) \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::f(a.c(i), (T)b); return r; }
#define CHAI_CL_LIFT2I(f)                                                                              \
template <class T, int N> __device__ __forceinline__ vec<T, N> f(const vec<T, N>& a, const vec<int, N>& b) \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::f(a.c(i), b.c(i)); return r; }                                  \
template <class T, int N> __device__ __forceinline__ vec<T, N> f(const vec<T, N>& a, int b)              \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::f(a.c(i), b); return r; }
#define CHAI_CL_LIFT3(f)                                                                               \
template <class T, int N>                                                                                \
__device__ __forceinline__ vec<T, N> f(const vec<T, N>& a, const vec<T, N>& b, const vec<T, N>& c)       \
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::f(a.c(i), b.c(i), c.c(i)); return r; }
CHAI_CL_LIFT1(acos) CHAI_CL_LIFT1(acosh) CHAI_CL_LIFT1(asin) CHAI_CL_LIFT1(asinh) CHAI_CL_LIFT1(atan)
CHAI_CL_LIFT1(atanh) CHAI_CL_LIFT1(cbrt) CHAI_CL_LIFT1(ceil) CHAI_CL_LIFT1(cos) CHAI_CL_LIFT1(cosh)
CHAI_CL_LIFT1(cospi) CHAI_CL_LIFT1(erf) CHAI_CL_LIFT1(erfc) CHAI_CL_LIFT1(exp) CHAI_CL_LIFT1(exp2)
CHAI_CL_LIFT1(exp10) CHAI_CL_LIFT1(expm1) CHAI_CL_LIFT1(fabs) CHAI_CL_LIFT1(floor) CHAI_CL_LIFT1(lgamma)
CHAI_CL_LIFT1(log) CHAI_CL_LIFT1(log10) CHAI_CL_LIFT1(log1p) CHAI_CL_LIFT1(log2) CHAI_CL_LIFT1(logb)
CHAI_CL_LIFT1(rint) CHAI_CL_LIFT1(round) CHAI_CL_LIFT1(rsqrt) CHAI_CL_LIFT1(sin) CHAI_CL_LIFT1(sinh)
CHAI_CL_LIFT1(sinpi) CHAI_CL_LIFT1(sqrt) CHAI_CL_LIFT1(tan) CHAI_CL_LIFT1(tanh) CHAI_CL_LIFT1(tgamma)
CHAI_CL_LIFT1(trunc) CHAI_CL_LIFT1(sign) CHAI_CL_LIFT1(degrees) CHAI_CL_LIFT1(radians) CHAI_CL_LIFT1(clz)
CHAI_CL_LIFT1(popcount)
CHAI_CL_LIFT2(atan2) CHAI_CL_LIFT2(copysign) CHAI_CL_LIFT2(fdim) CHAI_CL_LIFT2(fmax) CHAI_CL_LIFT2(fmin)
CHAI_CL_LIFT2(fmod) CHAI_CL_LIFT2(hypot) CHAI_CL_LIFT2(nextafter) CHAI_CL_LIFT2(pow) CHAI_CL_LIFT2(remainder)
CHAI_CL_LIFT2(rotate) CHAI_CL_LIFT2(mul_hi) CHAI_CL_LIFT2(mul24) CHAI_CL_LIFT2(hadd) CHAI_CL_LIFT2(rhadd)
CHAI_CL_LIFT2(add_sat) CHAI_CL_LIFT2(sub_sat)
CHAI_CL_LIFT2I(ldexp) CHAI_CL_LIFT2I(pown) CHAI_CL_LIFT2I(rootn)
CHAI_CL_LIFT3(fma) CHAI_CL_LIFT3(mad24)
#undef CHAI_CL_LIFT1
#undef CHAI_CL_LIFT2
#undef CHAI_CL_LIFT2I
#undef CHAI_CL_LIFT3
template <class T, int N> __device__ __forceinline__ vec<T, N> mad(const vec<T, N>& a, const vec<T, N>& b, const vec<T, N>& c)
{ return a * b + c; }
// min / max: y if y < x (resp. x < y), else x
template <class T, int N> __device__ __forceinline__ vec<T, N> min(const vec<T, N>& a, const vec<T, N>& b)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = b.c(i) < a.c(i) ? b.c(i) : a.c(i); return r; }
template <class T, int N> __device__ __forceinline__ vec<T, N> max(const vec<T, N>& a, const vec<T, N>& b)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = a.c(i) < b.c(i) ? b.c(i) : a.c(i); return r; }
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> min(const vec<T, N>& a, S b)
{ return min(a, vec<T, N>((T)b)); }
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> max(const vec<T, N>& a, S b)
{ return max(a, vec<T, N>((T)b)); }
template <class T, int N> __device__ __forceinline__ vec<T, N> clamp(const vec<T, N>& x, const vec<T, N>& lo, const vec<T, N>& hi)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::clamp(x.c(i), lo.c(i), hi.c(i)); return r; }
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> clamp(const vec<T, N>& x, S lo, S hi)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::clamp(x.c(i), (T)lo, (T)hi); return r; }
template <class T, int N> __device__ __forceinline__ vec<T, N> mix(const vec<T, N>& x, const vec<T, N>& y, const vec<T, N>& a)
{ return x + (y - x) * a; }
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> mix(const vec<T, N>& x, const vec<T, N>& y, S a)
{ return x + (y - x) * (T)a; }
template <class T, int N> __device__ __forceinline__ vec<T, N> step(const vec<T, N>& e, const vec<T, N>& x)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::step(e.c(i), x.c(i)); return r; }
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> step(S e, const vec<T, N>& x)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::step((T)e, x.c(i)); return r; }
template <class T, int N>
__device__ __forceinline__ vec<T, N> smoothstep(const vec<T, N>& e0, const vec<T, N>& e1, const vec<T, N>& x)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::smoothstep(e0.c(i), e1.c(i), x.c(i)); return r; }
template <class T, int N, class S> __device__ __forceinline__ if_num<S, vec<T, N>> smoothstep(S e0, S e1, const vec<T, N>& x)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::smoothstep((T)e0, (T)e1, x.c(i)); return r; }
template <class T, int N> __device__ __forceinline__ vec<utype<T>, N> abs(const vec<T, N>& a)
{ vec<utype<T>, N> r; CHAI_CL_FOR(N) r.c(i) = (utype<T>)(a.c(i) < 0 ? (utype<T>)0 - (utype<T>)a.c(i) : (utype<T>)a.c(i)); return r; }
template <class T, int N> __device__ __forceinline__ vec<utype<T>, N> abs_diff(const vec<T, N>& a, const vec<T, N>& b)
{ vec<utype<T>, N> r; CHAI_CL_FOR(N) r.c(i) = ::abs_diff(a.c(i), b.c(i)); return r; }
// relational built-ins: -1 / 0 per component
#define CHAI_CL_REL1(f, e)                                                                             \
template <class T, int N> __device__ __forceinline__ cvec<T, N> f(const vec<T, N>& a)                    \
{ cvec<T, N> r; CHAI_CL_FOR(N) { const T x = a.c(i); r.c(i) = (e) ? -1 : 0; } return r; }
CHAI_CL_REL1(isnan, x != x)
CHAI_CL_REL1(isinf, ::isinf(x))
CHAI_CL_REL1(isfinite, ::isfinite(x))
CHAI_CL_REL1(signbit, ::signbit(x))
CHAI_CL_REL1(isnormal, ::isfinite(x) && ::fabs(x) >= (sizeof(T) == 4 ? (T)0x1p-126 : (T)0x1p-1022))
#undef CHAI_CL_REL1
#define CHAI_CL_REL2(f, e)                                                                             \
template <class T, int N> __device__ __forceinline__ cvec<T, N> f(const vec<T, N>& a, const vec<T, N>& b) \
{ cvec<T, N> r; CHAI_CL_FOR(N) { const T x = a.c(i), y = b.c(i); r.c(i) = (e) ? -1 : 0; } return r; }
CHAI_CL_REL2(isequal, x == y) CHAI_CL_REL2(isnotequal, x != y) CHAI_CL_REL2(isgreater, x > y)
CHAI_CL_REL2(isgreaterequal, x >= y) CHAI_CL_REL2(isless, x < y) CHAI_CL_REL2(islessequal, x <= y)
CHAI_CL_REL2(islessgreater, x < y || x > y) CHAI_CL_REL2(isordered, x == x && y == y)
CHAI_CL_REL2(isunordered, x != x || y != y)
#undef CHAI_CL_REL2
template <class T, int N> __device__ __forceinline__ int any(const vec<T, N>& a)
{ bool r = false; CHAI_CL_FOR(N) r = r || msb(a.c(i)); return r; }
template <class T, int N> __device__ __forceinline__ int all(const vec<T, N>& a)
{ bool r = true; CHAI_CL_FOR(N) r = r && msb(a.c(i)); return r; }
template <class T, class U, int N>
__device__ __forceinline__ vec<T, N> select(const vec<T, N>& a, const vec<T, N>& b, const vec<U, N>& c)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = msb(c.c(i)) ? b.c(i) : a.c(i); return r; }
template <class T, int N>
__device__ __forceinline__ vec<T, N> bitselect(const vec<T, N>& a, const vec<T, N>& b, const vec<T, N>& c)
{ vec<T, N> r; CHAI_CL_FOR(N) r.c(i) = ::bitselect(a.c(i), b.c(i), c.c(i)); return r; }
// geometric built-ins (2, 3, 4 components)
template <class T, int N> __device__ __forceinline__ T dot(const vec<T, N>& a, const vec<T, N>& b)
{
    T s = a.c(0) * b.c(0);
    _Pragma("unroll") for (int i = 1; i < N; i++) s = s + a.c(i) * b.c(i);
    return s;
}
template <class T> __device__ __forceinline__ vec<T, 3> cross(const vec<T, 3>& a, const vec<T, 3>& b)
{ return vec<T, 3>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
template <class T> __device__ __forceinline__ vec<T, 4> cross(const vec<T, 4>& a, const vec<T, 4>& b)
{ return vec<T, 4>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, T(0)); }
template <class T, int N> __device__ __forceinline__ T length(const vec<T, N>& a) { return ::sqrt(dot(a, a)); }
template <class T, int N> __device__ __forceinline__ T distance(const vec<T, N>& a, const vec<T, N>& b) { return length(a - b); }
template <class T, int N> __device__ __forceinline__ vec<T, N> normalize(const vec<T, N>& a)
{
    const T l = length(a);
    return l == T(0) ? a : a / l;
}
// ---- images: an array bound to an image2d_t parameter is read as rows of
// 16-byte RGBA texels (4 x 32-bit channels; an f64 array holds 2 values per
// texel, read with read_imageui and as_double2)
struct image2d {
    unsigned char* p;
    int w, h;          // texels per row, rows
};
__device__ __forceinline__ int get_image_width(const image2d& im) { return im.w; }
__device__ __forceinline__ int get_image_height(const image2d& im) { return im.h; }
__device__ __forceinline__ vec<int, 2> get_image_dim(const image2d& im) { return vec<int, 2>(im.w, im.h); }
template <class T> __device__ __forceinline__ vec<T, 4> texel(const image2d& im, int i, int j)
{ return *reinterpret_cast<const vec<T, 4>*>(im.p + ((size_t)j * (size_t)im.w + (size_t)i) * 16); }
// a texel index under the sampler's addressing; -1 where CLK_ADDRESS_CLAMP
// reads the border colour.  Every other mode stays inside the image.
__device__ __forceinline__ int addr(int i, int w, unsigned smp)
{
    if ((smp & 14u) == CLK_ADDRESS_CLAMP) return (i < 0 || i >= w) ? -1 : i;
    return i < 0 ? 0 : (i >= w ? w - 1 : i);
}
template <class T> __device__ __forceinline__ vec<T, 4> fetch(const image2d& im, unsigned smp, int i, int j)
{
    const int a = addr(i, im.w, smp), b = addr(j, im.h, smp);
    if (a < 0 || b < 0) return vec<T, 4>(T(0));
    return texel<T>(im, a, b);
}
// normalized coordinate -> texel space, with the repeat modes' wrap
__device__ __forceinline__ float unnorm(float s, int w, unsigned smp)
{
    if (!(smp & 1u)) return s;
    const unsigned a = smp & 14u;
    if (a == CLK_ADDRESS_REPEAT) return (s - floorf(s)) * (float)w;
    if (a == CLK_ADDRESS_MIRRORED_REPEAT) {
        const float t = fabsf(s - 2.0f * rintf(0.5f * s));
        return t * (float)w;
    }
    return s * (float)w;
}
__device__ __forceinline__ int nearest(float u, int w, unsigned smp)
{
    int i = (int)floorf(u);
    const unsigned a = smp & 14u;
    if ((smp & 1u) && a == CLK_ADDRESS_REPEAT && i > w - 1) i -= w;
    if ((smp & 1u) && a == CLK_ADDRESS_MIRRORED_REPEAT && i > w - 1) i = w - 1;
    return i;
}
template <class T> __device__ __forceinline__ vec<T, 4> sample(const image2d& im, unsigned smp, const vec<float, 2>& c)
{
    const float u = unnorm(c.x, im.w, smp), v = unnorm(c.y, im.h, smp);
    if (!num<T>::fp || !(smp & CLK_FILTER_LINEAR)) return fetch<T>(im, smp, nearest(u, im.w, smp), nearest(v, im.h, smp));
    const float uu = u - 0.5f, vv = v - 0.5f;
    int i0 = (int)floorf(uu), j0 = (int)floorf(vv), i1 = i0 + 1, j1 = j0 + 1;
    const float a = uu - floorf(uu), b = vv - floorf(vv);
    const unsigned m = smp & 14u;
    if ((smp & 1u) && m == CLK_ADDRESS_REPEAT) {
        if (i0 < 0) i0 += im.w;
        if (i1 > im.w - 1) i1 -= im.w;
        if (j0 < 0) j0 += im.h;
        if (j1 > im.h - 1) j1 -= im.h;
    } else if ((smp & 1u) && m == CLK_ADDRESS_MIRRORED_REPEAT) {
        i0 = i0 < 0 ? 0 : i0;
        i1 = i1 > im.w - 1 ? im.w - 1 : i1;
        j0 = j0 < 0 ? 0 : j0;
        j1 = j1 > im.h - 1 ? im.h - 1 : j1;
    }
    const vec<T, 4> t00 = fetch<T>(im, smp, i0, j0), t10 = fetch<T>(im, smp, i1, j0);
    const vec<T, 4> t01 = fetch<T>(im, smp, i0, j1), t11 = fetch<T>(im, smp, i1, j1);
    return (T)((1 - a) * (1 - b)) * t00 + (T)(a * (1 - b)) * t10 + (T)((1 - a) * b) * t01 + (T)(a * b) * t11;
}
__device__ __forceinline__ vec<float, 4> read_imagef(const image2d& im, unsigned smp, const vec<int, 2>& c)
{ return fetch<float>(im, smp, c.x, c.y); }
__device__ __forceinline__ vec<float, 4> read_imagef(const image2d& im, unsigned smp, const vec<float, 2>& c)
{ return sample<float>(im, smp, c); }
__device__ __forceinline__ vec<float, 4> read_imagef(const image2d& im, const vec<int, 2>& c)
{ return fetch<float>(im, CLK_ADDRESS_CLAMP_TO_EDGE, c.x, c.y); }
__device__ __forceinline__ vec<int, 4> read_imagei(const image2d& im, unsigned smp, const vec<int, 2>& c)
{ return fetch<int>(im, smp, c.x, c.y); }
__device__ __forceinline__ vec<int, 4> read_imagei(const image2d& im, unsigned smp, const vec<float, 2>& c)
{ return sample<int>(im, smp, c); }
__device__ __forceinline__ vec<int, 4> read_imagei(const image2d& im, const vec<int, 2>& c)
{ return fetch<int>(im, CLK_ADDRESS_CLAMP_TO_EDGE, c.x, c.y); }
__device__ __forceinline__ vec<unsigned, 4> read_imageui(const image2d& im, unsigned smp, const vec<int, 2>& c)
{ return fetch<unsigned>(im, smp, c.x, c.y); }
__device__ __forceinline__ vec<unsigned, 4> read_imageui(const image2d& im, unsigned smp, const vec<float, 2>& c)
{ return sample<unsigned>(im, smp, c); }
__device__ __forceinline__ vec<unsigned, 4> read_imageui(const image2d& im, const vec<int, 2>& c)
{ return fetch<unsigned>(im, CLK_ADDRESS_CLAMP_TO_EDGE, c.x, c.y); }
// writes outside the image are dropped
template <class T> __device__ __forceinline__ void store_texel(const image2d& im, const vec<int, 2>& c, const vec<T, 4>& v)
{
    if (c.x < 0 || c.y < 0 || c.x >= im.w || c.y >= im.h) return;
    *reinterpret_cast<vec<T, 4>*>(im.p + ((size_t)c.y * (size_t)im.w + (size_t)c.x) * 16) = v;
}
__device__ __forceinline__ void write_imagef(const image2d& im, const vec<int, 2>& c, const vec<float, 4>& v) { store_texel(im, c, v); }
__device__ __forceinline__ void write_imagei(const image2d& im, const vec<int, 2>& c, const vec<int, 4>& v) { store_texel(im, c, v); }
__device__ __forceinline__ void write_imageui(const image2d& im, const vec<int, 2>& c, const vec<unsigned, 4>& v) { store_texel(im, c, v); }
}  // namespace chai_cl
typedef chai_cl::image2d image2d_t;
// vloadN / vstoreN: N components at p + i*N (element alignment; one vector
// access where the address is aligned to the vector)
#define CHAI_CL_VLOAD(N)                                                                               \
template <class T> __device__ __forceinline__ chai_cl::vec<T, N> vload##N(size_t i, const T* p)          \
{                                                                                                        \
    const T* q = p + i * N;                                                                              \
    if (N != 3 && ((size_t)q & (sizeof(chai_cl::vec<T, N>) - 1)) == 0)                                  \
        return *reinterpret_cast<const chai_cl::vec<T, N>*>(q);                                          \
    chai_cl::vec<T, N> r;                                                                                \
    _Pragma("unroll") for (int k = 0; k < N; k++) r.c(k) = q[k];                                         \
    return r;                                                                                            \
}                                                                                                        \
template <class T> __device__ __forceinline__ void vstore##N(const chai_cl::vec<T, N>& v, size_t i, T* p) \
{                                                                                                        \
    T* q = p + i * N;                                                                                    \
    if (N != 3 && ((size_t)q & (sizeof(chai_cl::vec<T, N>) - 1)) == 0) {                                 \
        *reinterpret_cast<chai_cl::vec<T, N>*>(q) = v;                                                   \
        return;                                                                                          \
    }                                                                                                    \
    _Pragma("unroll") for (int k = 0; k < N; k++) q[k] = v.c(k);                                         \
}
CHAI_CL_VLOAD(2) CHAI_CL_VLOAD(3) CHAI_CL_VLOAD(4) CHAI_CL_VLOAD(8) CHAI_CL_VLOAD(16)
#undef CHAI_CL_VLOAD
// ---- half as a storage format (OpenCL 1.2 without cl_khr_fp16): vload_half*
// widen IEEE binary16 to float, vstore_half* round float / double to it
// (_rte the default, _rtz, _rtp, _rtn) with the PTX conversions
namespace chai_cl {
struct half_t { unsigned short bits; };
__device__ __forceinline__ float h2f(unsigned short h) { float f; asm("cvt.f32.f16 %0, %1;" : "=f"(f) : "h"(h)); return f; }
template <int M> __device__ __forceinline__ unsigned short f2h(float f)
{
    unsigned short h;
    if (M == 2) asm("cvt.rz.f16.f32 %0, %1;" : "=h"(h) : "f"(f));
    else if (M == 3) asm("cvt.rp.f16.f32 %0, %1;" : "=h"(h) : "f"(f));
    else if (M == 4) asm("cvt.rm.f16.f32 %0, %1;" : "=h"(h) : "f"(f));
    else asm("cvt.rn.f16.f32 %0, %1;" : "=h"(h) : "f"(f));
    return h;
}
template <int M> __device__ __forceinline__ unsigned short f2h(double f)
{
    unsigned short h;
    if (M == 2) asm("cvt.rz.f16.f64 %0, %1;" : "=h"(h) : "d"(f));
    else if (M == 3) asm("cvt.rp.f16.f64 %0, %1;" : "=h"(h) : "d"(f));
    else if (M == 4) asm("cvt.rm.f16.f64 %0, %1;" : "=h"(h) : "d"(f));
    else asm("cvt.rn.f16.f64 %0, %1;" : "=h"(h) : "d"(f));
    return h;
}
}  // namespace chai_cl
typedef chai_cl::half_t half;
__device__ __forceinline__ float vload_half(size_t i, const half* p) { return chai_cl::h2f(p[i].bits); }
#define CHAI_CL_VLOAD_HALF(N, A)                                                                         \
__device__ __forceinline__ chai_cl::vec<float, N> vload##A##_half##N(size_t i, const half* p)            \
{ chai_cl::vec<float, N> r; _Pragma("unroll") for (int k = 0; k < N; k++) r.c(k) = chai_cl::h2f(p[i * (N == 3 && #A[0] ? 4 : N) + k].bits); return r; }
CHAI_CL_VLOAD_HALF(2, ) CHAI_CL_VLOAD_HALF(3, ) CHAI_CL_VLOAD_HALF(4, ) CHAI_CL_VLOAD_HALF(8, ) CHAI_CL_VLOAD_HALF(16, )
CHAI_CL_VLOAD_HALF(2, a) CHAI_CL_VLOAD_HALF(3, a) CHAI_CL_VLOAD_HALF(4, a) CHAI_CL_VLOAD_HALF(8, a) CHAI_CL_VLOAD_HALF(16, a)
#undef CHAI_CL_VLOAD_HALF
#define CHAI_CL_VSTORE_HALF1(SUF, M)                                                                     \
__device__ __forceinline__ void vstore_half##SUF(float d, size_t i, half* p) { p[i].bits = chai_cl::f2h<M>(d); } \
__device__ __forceinline__ void vstore_half##SUF(double d, size_t i, half* p) { p[i].bits = chai_cl::f2h<M>(d); }
CHAI_CL_VSTORE_HALF1(, 1) CHAI_CL_VSTORE_HALF1(_rte, 1) CHAI_CL_VSTORE_HALF1(_rtz, 2) CHAI_CL_VSTORE_HALF1(_rtp, 3)
CHAI_CL_VSTORE_HALF1(_rtn, 4)
#undef CHAI_CL_VSTORE_HALF1
#define CHAI_CL_VSTORE_HALFN(N, A, SUF, M)                                                              \
template <class T> __device__ __forceinline__ void vstore##A##_half##N##SUF(const chai_cl::vec<T, N>& v, size_t i, half* p) \
{ _Pragma("unroll") for (int k = 0; k < N; k++) p[i * (N == 3 && #A[0] ? 4 : N) + k].bits = chai_cl::f2h<M>(v.c(k)); }
#define CHAI_CL_VSTORE_HALF_MODES(N, A)                                                                  \
CHAI_CL_VSTORE_HALFN(N, A, , 1) CHAI_CL_VSTORE_HALFN(N, A, _rte, 1) CHAI_CL_VSTORE_HALFN(N, A, _rtz, 2)   \
CHAI_CL_VSTORE_HALFN(N, A, _rtp, 3) CHAI_CL_VSTORE_HALFN(N, A, _rtn, 4)
CHAI_CL_VSTORE_HALF_MODES(2, ) CHAI_CL_VSTORE_HALF_MODES(3, ) CHAI_CL_VSTORE_HALF_MODES(4, )
CHAI_CL_VSTORE_HALF_MODES(8, ) CHAI_CL_VSTORE_HALF_MODES(16, )
CHAI_CL_VSTORE_HALF_MODES(2, a) CHAI_CL_VSTORE_HALF_MODES(3, a) CHAI_CL_VSTORE_HALF_MODES(4, a)
CHAI_CL_VSTORE_HALF_MODES(8, a) CHAI_CL_VSTORE_HALF_MODES(16, a)
#undef CHAI_CL_VSTORE_HALF_MODES
#undef CHAI_CL_VSTORE_HALFN
// ---- program text
)cl";

namespace {

struct Tok {
    enum Kind { IDENT, OTHER } kind;
    std::string text;
};

// identifiers, and everything else (punctuation, numbers, white space,
// comments, literals) as opaque runs
std::vector<Tok> tokenize(const std::string& s)
{
    std::vector<Tok> out;
    size_t i = 0;
    auto other = [&](size_t a, size_t b) {
        if (!out.empty() && out.back().kind == Tok::OTHER) out.back().text.append(s, a, b - a);
        else out.push_back({Tok::OTHER, s.substr(a, b - a)});
    };
    while (i < s.size()) {
        const char c = s[i];
        if (std::isalpha((unsigned char)c) || c == '_') {
            size_t j = i + 1;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) j++;
            out.push_back({Tok::IDENT, s.substr(i, j - i)});
            i = j;
        } else if (std::isdigit((unsigned char)c)) {
            size_t j = i + 1;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '.' || s[j] == '_')) j++;
            other(i, j);
            i = j;
        } else if (c == '/' && i + 1 < s.size() && s[i + 1] == '/') {
            size_t j = s.find('\n', i);
            j = j == std::string::npos ? s.size() : j;
            other(i, j);
            i = j;
        } else if (c == '/' && i + 1 < s.size() && s[i + 1] == '*') {
            size_t j = s.find("*/", i + 2);
            j = j == std::string::npos ? s.size() : j + 2;
            other(i, j);
            i = j;
        } else if (c == '"' || c == '\'') {
            size_t j = i + 1;
            while (j < s.size() && s[j] != c) j += (s[j] == '\\') ? 2 : 1;
            j = std::min(s.size(), j + 1);
            other(i, j);
            i = j;
        } else {
            other(i, i + 1);
            i++;
        }
    }
    return out;
}

bool is_kernel_kw(const std::string& t) { return t == "__kernel" || t == "kernel"; }
bool names(const std::vector<Tok>& p, const char* word)
{
    for (const Tok& x : p)
        if (x.kind == Tok::IDENT && x.text == word) return true;
    return false;
}
bool is_local_kw(const std::string& t) { return t == "__local" || t == "local"; }
bool is_access_qualifier(const std::string& t)
{
    return t == "__read_only" || t == "read_only" || t == "__write_only" || t == "write_only" ||
           t == "__read_write" || t == "read_write";
}

// OpenCL scalar names -> the C++ type of a vector component
const char* cl_elem(const std::string& s)
{
    static const char* const k[][2] = {{"char", "signed char"}, {"uchar", "unsigned char"}, {"short", "short"},
                                       {"ushort", "unsigned short"}, {"int", "int"}, {"uint", "unsigned int"},
                                       {"long", "long long"}, {"ulong", "unsigned long long"},
                                       {"float", "float"}, {"double", "double"}};
    for (const auto& e : k)
        if (s == e[0]) return e[1];
    return nullptr;
}

// "float4" -> ("float", 4); false unless `w` names an OpenCL vector type
bool vec_type(const std::string& w, std::string& elem, int& n)
{
    size_t d = w.size();
    while (d > 0 && std::isdigit((unsigned char)w[d - 1])) d--;
    if (d == 0 || d == w.size()) return false;
    const std::string count = w.substr(d);
    if (count != "2" && count != "3" && count != "4" && count != "8" && count != "16") return false;
    const char* e = cl_elem(w.substr(0, d));
    if (!e) return false;
    elem = e;
    n = std::stoi(count);
    return true;
}

std::string vec_cpp(const std::string& elem, int n) { return "chai_cl::vec<" + elem + ", " + std::to_string(n) + ">"; }

// convert_<type>[N][_sat][_rte|_rtz|_rtp|_rtn] -> chai_cl::convert<component, N, sat, mode>
bool convert_name(const std::string& w, std::string& out)
{
    if (w.compare(0, 8, "convert_") != 0) return false;
    std::string rest = w.substr(8);
    int mode = 0;
    static const char* const modes[] = {"_rte", "_rtz", "_rtp", "_rtn"};
    for (int m = 0; m < 4; m++) {
        if (rest.size() > 4 && rest.compare(rest.size() - 4, 4, modes[m]) == 0) {
            mode = m + 1;
            rest.resize(rest.size() - 4);
            break;
        }
    }
    int sat = 0;
    if (rest.size() > 4 && rest.compare(rest.size() - 4, 4, "_sat") == 0) {
        sat = 1;
        rest.resize(rest.size() - 4);
    }
    std::string elem;
    int n = 1;
    if (!vec_type(rest, elem, n)) {
        const char* e = cl_elem(rest);
        if (!e) return false;
        elem = e;
    }
    out = "chai_cl::convert<" + elem + ", " + std::to_string(n) + ", " + std::to_string(sat) + ", " +
          std::to_string(mode) + ">";
    return true;
}

// as_<type>[N] -> chai_cl::as_type<type>
bool as_name(const std::string& w, std::string& out)
{
    if (w.compare(0, 3, "as_") != 0) return false;
    const std::string rest = w.substr(3);
    std::string elem;
    int n = 0;
    if (vec_type(rest, elem, n)) {
        out = "chai_cl::as_type<" + vec_cpp(elem, n) + ">";
        return true;
    }
    const char* e = cl_elem(rest);
    if (!e) return false;
    out = std::string("chai_cl::as_type<") + e + ">";
    return true;
}

// The components a swizzle selects (.xy, .s01, .sF) or, in `special`, one of
// lo / hi / even / odd.  Single x / y / z / w letters are real members and
// are not swizzles here.
bool swizzle(const std::string& w, std::vector<int>& idx, std::string& special)
{
    idx.clear();
    special.clear();
    if (w == "lo" || w == "hi" || w == "even" || w == "odd") {
        special = w;
        return true;
    }
    if ((w[0] == 's' || w[0] == 'S') && w.size() >= 2 && w.size() <= 17) {
        for (size_t k = 1; k < w.size(); k++) {
            const char c = w[k];
            const int v = std::isdigit((unsigned char)c) ? c - '0'
                        : (c >= 'a' && c <= 'f')         ? c - 'a' + 10
                        : (c >= 'A' && c <= 'F')         ? c - 'A' + 10
                                                          : -1;
            if (v < 0) return false;
            idx.push_back(v);
        }
        return true;
    }
    if (w.size() < 2 || w.size() > 4) return false;
    static const char kXYZW[] = "xyzw";
    for (char c : w) {
        const char* p = c ? std::strchr(kXYZW, c) : nullptr;
        if (!p) return false;
        idx.push_back((int)(p - kXYZW));
    }
    return true;
}

// Bytes of one element of a __local parameter's declared type (after the
// vector rewrite); 0 when the type is not an OpenCL scalar or vector type.
size_t local_elem_bytes(const std::string& type)
{
    static const std::pair<const char*, size_t> scalars[] = {
        {"char", 1}, {"signed char", 1}, {"uchar", 1}, {"unsigned char", 1}, {"short", 2}, {"ushort", 2},
        {"unsigned short", 2}, {"int", 4}, {"uint", 4}, {"unsigned", 4}, {"unsigned int", 4}, {"float", 4},
        {"long", 8}, {"ulong", 8}, {"unsigned long", 8}, {"long long", 8}, {"unsigned long long", 8},
        {"double", 8}, {"size_t", 8}};
    for (const auto& e : scalars)
        if (type == e.first) return e.second;
    const std::string head = "chai_cl::vec<";
    if (type.compare(0, head.size(), head) != 0 || type.back() != '>') return 0;
    const size_t comma = type.rfind(',');
    if (comma == std::string::npos) return 0;
    const size_t eb = local_elem_bytes(type.substr(head.size(), comma - head.size()));
    const int n = std::atoi(type.c_str() + comma + 1);
    return eb * (size_t)(n == 3 ? 4 : n);
}

// true when the token after position i starts an assignment (=, op=, ++, --)
bool assigned_next(const std::vector<Tok>& t, size_t i)
{
    if (i + 1 >= t.size() || t[i + 1].kind != Tok::OTHER) return false;
    const std::string& s = t[i + 1].text;
    const size_t p = s.find_first_not_of(" \t\r\n");
    if (p == std::string::npos) return false;
    static const char* const ops[] = {"<<=", ">>=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "++", "--"};
    for (const char* o : ops)
        if (s.compare(p, std::strlen(o), o) == 0) return true;
    return s[p] == '=' && (p + 1 >= s.size() || s[p + 1] != '=');
}

// The rewrites that need no type information: vector type names, vector
// literals (floatN)(...), convert_ / as_ names, and -- only in a program that
// names a vector type, since .lo / .hi / .sN could otherwise be members of a
// struct -- swizzles after '.' or '->'.
void rewrite_vectors(std::vector<Tok>& t)
{
    bool vectors = false;
    for (const Tok& x : t) {
        std::string e;
        int n = 0;
        if (x.kind == Tok::IDENT && (vec_type(x.text, e, n) || x.text == "image2d_t" ||
                                     x.text.compare(0, 5, "vload") == 0 || x.text.compare(0, 6, "vstore") == 0)) {
            vectors = true;
            break;
        }
    }
    static const char* const ws = " \t\r\n";
    for (size_t i = 0; i < t.size(); i++) {
        if (t[i].kind != Tok::IDENT) continue;
        std::string& w = t[i].text;
        std::string elem, cpp;
        int n = 0;
        if (vec_type(w, elem, n)) {
            const std::string type = vec_cpp(elem, n);
            if (i > 0 && i + 1 < t.size() && t[i - 1].kind == Tok::OTHER && t[i + 1].kind == Tok::OTHER) {
                std::string& pre = t[i - 1].text;
                std::string& post = t[i + 1].text;
                const size_t a = pre.find_last_not_of(ws);
                const size_t b = post.find_first_not_of(ws);
                const size_t c = b == std::string::npos ? b : post.find_first_not_of(ws, b + 1);
                if (a != std::string::npos && pre[a] == '(' && b != std::string::npos && post[b] == ')' &&
                    c != std::string::npos && post[c] == '(') {
                    pre.erase(a);
                    post.erase(0, c);
                    w = "chai_cl::make<" + type + ">";
                    continue;
                }
            }
            w = type;
        } else if (convert_name(w, cpp) || as_name(w, cpp)) {
            w = cpp;
        } else if (vectors && i > 0 && t[i - 1].kind == Tok::OTHER) {
            const std::string& pre = t[i - 1].text;
            const size_t a = pre.find_last_not_of(ws);
            const bool dot = a != std::string::npos && pre[a] == '.' && (a == 0 || pre[a - 1] != '.');
            const bool arrow = a != std::string::npos && a > 0 && pre[a] == '>' && pre[a - 1] == '-';
            if (!dot && !arrow) continue;
            std::vector<int> idx;
            std::string special;
            if (!swizzle(w, idx, special)) continue;
            const bool lv = assigned_next(t, i);
            if (!special.empty()) {
                w = "chai_" + special + (lv ? "_l()" : "()");
            } else if (idx.size() == 1) {
                w = "chai_sw1<" + std::to_string(idx[0]) + ">()";
            } else {
                std::string s = lv ? "chai_swl<" : "chai_swr<";
                for (size_t k = 0; k < idx.size(); k++) s += (k ? "," : "") + std::to_string(idx[k]);
                w = s + ">()";
            }
        }
    }
}

}  // namespace

// `local_counts[i]`: elements of the i-th argument of kernel `name` when it is
// a __local pointer (0 otherwise); each is sized by its declared element type
// and `*local_bytes`, when given, receives the dynamic shared memory they
// take.  `image_args`, when given, receives one flag per parameter of kernel
// `name`: 1 for an image2d_t parameter, which takes two launch arguments (the
// texel pointer, then width | height << 32).
int opencl_to_cuda(const std::string& src, const std::string& name, const std::vector<size_t>& local_counts,
                   int work_dim, std::string& out, std::string& err, std::vector<char>* image_args,
                   size_t* local_bytes)
{
    std::vector<Tok> t = tokenize(src);
    rewrite_vectors(t);
    std::ostringstream os;
    os << "#define CHAI_CL_WORK_DIM " << work_dim << "\n" << kOpenCLPrelude << kOpenCLVectors;
    bool found = false;
    for (size_t i = 0; i < t.size(); i++) {
        if (t[i].kind != Tok::IDENT) {
            os << t[i].text;
            continue;
        }
        const std::string& w = t[i].text;
        if (is_kernel_kw(w)) {
            // __kernel void NAME ( params ) {
            size_t j = i + 1;
            auto next_ident = [&](size_t& k) -> int {
                while (k < t.size() && t[k].kind == Tok::OTHER) {
                    for (char ch : t[k].text)
                        if (!std::isspace((unsigned char)ch)) return -1;
                    k++;
                }
                return k < t.size() ? (int)k : -1;
            };
            int kv = next_ident(j);
            // __attribute__((...)) between __kernel and void (dropped), as the
            // reference's parser skips every token up to "void"
            // (api/ProgramCL.cpp:156-177)
            while (kv >= 0 && t[kv].text == "__attribute__") {
                size_t q = (size_t)kv + 1;
                int depth = 0;
                bool opened = false, closed = false;
                for (; q < t.size() && !closed; q++) {
                    if (t[q].kind != Tok::OTHER) continue;
                    const std::string& x = t[q].text;
                    for (size_t c = 0; c < x.size(); c++) {
                        if (x[c] == '(') { depth++; opened = true; }
                        if (x[c] == ')' && --depth == 0 && opened) {
                            if (x.find_first_not_of(" \t\r\n", c + 1) != std::string::npos) {
                                err = "inline kernel: unexpected text after __attribute__";
                                return -1;
                            }
                            closed = true;
                            break;
                        }
                    }
                }
                if (!closed) { err = "inline kernel: unbalanced __attribute__"; return -1; }
                j = q;
                kv = next_ident(j);
            }
            if (kv < 0 || t[kv].text != "void") { err = "inline kernel: expected void after __kernel"; return -1; }
            j = (size_t)kv + 1;
            int kn = next_ident(j);
            if (kn < 0) { err = "inline kernel: missing kernel name"; return -1; }
            const std::string kname = t[kn].text;
            // parameters: tokens up to the matching ')'
            size_t k = (size_t)kn + 1;
            std::string pre;          // text between name and '('
            while (k < t.size() && !(t[k].kind == Tok::OTHER && t[k].text.find('(') != std::string::npos)) pre += t[k++].text;
            if (k >= t.size()) { err = "inline kernel: missing parameter list"; return -1; }
            const size_t lp = t[k].text.find('(');
            const std::string params_before = t[k].text.substr(0, lp);
            std::vector<Tok> plist;
            int depth = 1;
            std::string tail;        // text after the closing ')' within its run
            auto walk = [&](const std::string& txt) -> bool {
                std::string cur;
                for (size_t p = 0; p < txt.size(); p++) {
                    const char ch = txt[p];
                    if (ch == '(') depth++;
                    if (ch == ')' && --depth == 0) {
                        if (!cur.empty()) plist.push_back({Tok::OTHER, cur});
                        tail = txt.substr(p + 1);
                        return true;
                    }
                    cur += ch;
                }
                if (!cur.empty()) plist.push_back({Tok::OTHER, cur});
                return false;
            };
            bool closed = walk(t[k].text.substr(lp + 1));
            k++;
            while (!closed && k < t.size()) {
                if (t[k].kind == Tok::IDENT) plist.push_back(t[k]);
                else closed = walk(t[k].text);
                k++;
            }
            if (!closed) { err = "inline kernel: unbalanced parameter list"; return -1; }
            // the rest of the run holding ')' is processed next
            k--;
            t[k] = {Tok::OTHER, tail};
            // rewrite the parameters one by one (split at top-level commas)
            std::vector<std::vector<Tok>> params(1);
            for (const Tok& x : plist) {
                if (x.kind == Tok::IDENT) { params.back().push_back(x); continue; }
                std::string cur;
                for (char ch : x.text) {
                    if (ch == ',') {
                        if (!cur.empty()) params.back().push_back({Tok::OTHER, cur});
                        cur.clear();
                        params.emplace_back();
                    } else {
                        cur += ch;
                    }
                }
                if (!cur.empty()) params.back().push_back({Tok::OTHER, cur});
            }
            std::ostringstream inject, img_inject;
            size_t offset = 0;
            const bool called = kname == name;
            if (called) {
                found = true;
                if (image_args) image_args->assign(params.size(), 0);
            }
            std::ostringstream plist_out;
            for (size_t pi = 0; pi < params.size(); pi++) {
                bool local = false;
                std::string last_ident, type;
                std::ostringstream pout;
                for (const Tok& x : params[pi]) {
                    if (x.kind == Tok::IDENT) {
                        if (is_local_kw(x.text)) { local = true; continue; }
                        if (is_access_qualifier(x.text)) continue;
                        if (x.text == "__global" || x.text == "global" || x.text == "__private" ||
                            x.text == "private")
                            continue;
                        if (x.text == "__constant" || x.text == "constant") { pout << "const"; continue; }
                        if (!last_ident.empty() && last_ident != "const" && last_ident != "volatile" &&
                            last_ident != "restrict")
                            type += (type.empty() ? "" : " ") + last_ident;
                        last_ident = x.text;
                        pout << x.text;
                    } else {
                        pout << x.text;
                    }
                }
                if (names(params[pi], "image3d_t")) {
                    err = "inline kernel: image3d_t arguments are not supported";
                    return -1;
                }
                if (names(params[pi], "sampler_t")) {
                    err = "inline kernel: sampler_t arguments are not supported (declare the sampler in the program)";
                    return -1;
                }
                if (names(params[pi], "image2d_t")) {
                    // the array's storage as rows of 16-byte texels: pointer + packed extent
                    const std::string& v = last_ident;
                    pout.str("");
                    pout << "unsigned char* chai_img_" << v << ", long long chai_imgd_" << v;
                    img_inject << " const chai_cl::image2d " << v << " = {chai_img_" << v << ", (int)(chai_imgd_" << v
                               << " & 0xffffffffLL), (int)(chai_imgd_" << v << " >> 32)};";
                    if (called && image_args) (*image_args)[pi] = 1;
                }
                if (local && called) {
                    const size_t count = pi < local_counts.size() ? local_counts[pi] : 0;
                    const size_t eb = local_elem_bytes(type);
                    if (eb == 0) {
                        err = "inline kernel: __local parameter " + last_ident + " has an element type of unknown size";
                        return -1;
                    }
                    if (count > (size_t)227 * 1024) {
                        err = "inline kernel: __local memory above 227 KB";
                        return -1;
                    }
                    inject << " " << last_ident << " = reinterpret_cast<" << type << "*>(chai_cl_lmem + " << offset
                           << ");";
                    offset += (count * eb + 15) & ~size_t(15);
                }
                plist_out << (pi ? "," : "") << pout.str();
            }
            if (called && local_bytes) *local_bytes = offset;
            os << "extern \"C\" __global__ void " << kname << pre << params_before << "(" << plist_out.str() << ")";
            // body: copy up to and including the opening '{', then inject
            while (k < t.size()) {
                if (t[k].kind == Tok::OTHER) {
                    const size_t b = t[k].text.find('{');
                    if (b != std::string::npos) {
                        os << t[k].text.substr(0, b + 1);
                        if (called && offset)
                            os << " extern __shared__ __align__(16) unsigned char chai_cl_lmem[];" << inject.str();
                        os << img_inject.str();
                        t[k].text = t[k].text.substr(b + 1);
                        break;
                    }
                }
                os << t[k].text;
                k++;
            }
            i = k - 1;      // resume with the remainder of the run holding '{'
            continue;
        }
        if (w == "__global" || w == "global" || w == "__private" || w == "private") continue;
        if (is_access_qualifier(w)) continue;
        if (w == "__constant" || w == "constant") { os << "const"; continue; }
        if (is_local_kw(w)) { os << "__shared__"; continue; }
        os << w;
    }
    if (!found) { err = "inline kernel: no __kernel named " + name; return -1; }
    out = os.str();
    return 0;
}

// Launch the inline kernel of node i: compile its program (cached by text),
// bind the arrays' storage, the scalars and the __local sizes, run it over the
// caller's NDRange.
int Translator::emit_inline(int i)
{
    const Node& nd = nodes_[i];
    const chai_inline_kernel& k = kernels_[nd.buffer];
    const bool two_d = k.global_size[1] != 0;
    for (int d = 0; d < (two_d ? 2 : 1); d++) {
        if (k.local_size[d] == 0 || k.global_size[d] % k.local_size[d] != 0)
            return fail(CHAI_ERR_INVALID, "inline kernel: local size must divide the global size");
    }
    const uint64_t lx = k.local_size[0], ly = two_d ? k.local_size[1] : 1;
    if (lx * ly > 1024) return fail(CHAI_ERR_INVALID, "inline kernel: more than 1024 work items per group");
    std::vector<size_t> lcount(k.n_args, 0);
    size_t smem = 0;
    for (uint32_t a = 0; a < k.n_args; a++) {
        const chai_kernel_arg& g = k.args[a];
        if (g.kind == CHAI_KARG_LOCAL) {
            // an element count; the kernel's declared element type sizes it
            if (!(g.value >= 0 && g.value <= 227.0 * 1024))
                return fail(CHAI_ERR_INVALID, "inline kernel: __local size out of range");
            lcount[a] = (size_t)g.value;
        } else if (g.kind != CHAI_KARG_ARRAY && g.kind != CHAI_KARG_SCALAR) {
            return fail(CHAI_ERR_INVALID, "inline kernel: argument kind");
        }
    }
    std::string cuda, err;
    std::vector<char> images;
    if (opencl_to_cuda(k.source, k.name, lcount, two_d ? 2 : 1, cuda, err, &images, &smem))
        return fail(CHAI_ERR_INVALID, err);
    if (smem > 227 * 1024) return fail(CHAI_ERR_INVALID, "inline kernel: __local memory above 227 KB");
    // an image2d_t argument: rows of whole 16-byte RGBA texels over one slot
    for (uint32_t a = 0, m = 0; a < k.n_args; a++) {
        if (k.args[a].kind != CHAI_KARG_ARRAY) continue;
        const Node& v = nodes_[nd.kids[m++]];
        if (a >= images.size() || !images[a]) continue;
        const uint64_t row = v.W * (uint64_t)prec_bytes(v.prec);
        if (v.slots != 1 || row % 16 != 0 || row / 16 > 0x7fffffffull || v.H > 0x7fffffffull)
            return fail(CHAI_ERR_INVALID, "inline kernel: an image2d_t argument needs a one-slot array whose rows "
                                          "are whole 16-byte texels");
    }
    last_source = cuda;
    all_sources += cuda;
    void* fn = nullptr;
    int st = ctx_->jit->get(cuda, k.name, &fn);
    if (st) return st;
    if (dry_) return CHAI_OK;
    Step ks;
    ks.kind = Step::KERNEL;
    ks.fn = fn;
    ks.grid = dim3((unsigned)(k.global_size[0] / lx), (unsigned)(two_d ? k.global_size[1] / ly : 1), 1);
    ks.block = dim3((unsigned)lx, (unsigned)ly, 1);
    ks.smem = smem;
    size_t m = 0;
    for (uint32_t a = 0; a < k.n_args; a++) {
        const chai_kernel_arg& g = k.args[a];
        Step::Arg arg;
        if (g.kind == CHAI_KARG_ARRAY) {
            const Node& v = nodes_[nd.kids[m++]];
            if (!v.dev) return fail(CHAI_ERR_INVALID, "inline kernel: array argument without storage");
            arg.kind = Step::Arg::PTR;
            arg.r = ref_of(v.dev);
            if (a < images.size() && images[a]) {
                // image2d_t: the storage pointer, then texels per row | rows << 32
                const uint64_t row = v.W * (uint64_t)prec_bytes(v.prec);
                if (((uintptr_t)v.dev & 15) != 0)
                    return fail(CHAI_ERR_INVALID, "inline kernel: image2d_t storage is not 16-byte aligned");
                ks.args.push_back(arg);
                Step::Arg extent;
                extent.kind = Step::Arg::I64;
                extent.v = (long long)((row / 16) | (v.H << 32));
                ks.args.push_back(extent);
                continue;
            }
        } else if (g.kind == CHAI_KARG_LOCAL) {
            arg.kind = Step::Arg::PTR;      // set by the kernel body to its slice of shared memory
        } else {
            arg.kind = Step::Arg::I64;      // the argument's bytes at the start of the slot
            long long bits = 0;
            if (g.prec == CHAI_F32) {
                const float f = (float)g.value;
                memcpy(&bits, &f, 4);
            } else if (g.prec == CHAI_F64) {
                memcpy(&bits, &g.value, 8);
            } else if (g.prec == CHAI_I32) {
                const int32_t v32 = (int32_t)(int64_t)g.value;
                memcpy(&bits, &v32, 4);
            } else {
                const uint32_t v32 = (uint32_t)(int64_t)g.value;
                memcpy(&bits, &v32, 4);
            }
            arg.v = bits;
        }
        ks.args.push_back(arg);
    }
    st = exec(ks);
    if (st) return st;
    kernels_launched++;
    return CHAI_OK;
}

}  // namespace chai
