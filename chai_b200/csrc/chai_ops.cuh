// Element operations of chai traces for sm_100a: one device function per
// bytecode opcode (bytecode/ByteCodes.hpp numbers), with the value semantics
// of the reference interpreter's scalar functors (misc/SimpleFun1.cpp,
// misc/SimpleFun2.cpp, misc/SimpleFun3.cpp): predicates give 1 or 0 in the
// operation's precision, max/min are `a < b ? b : a` / `a < b ? a : b`,
// saturating and 24-bit integer ops follow the interpreter's 64-bit
// arithmetic, the *pi variants divide by pi.  The precision of a two- or
// three-operand op is the widest operand precision (interp/InterpFun2.cpp:21,
// interp/InterpFun3.cpp:23); operands are converted to it before the op.
//
// Embedded verbatim into every runtime-compiled trace kernel (and usable by
// static kernels).
#pragma once
#ifndef CHAI_OPS_CUH
#define CHAI_OPS_CUH

namespace chai_ops {

typedef unsigned int u32;
typedef int i32;

#define CHAI_PI 3.14159265358979323846

// ---------------------------------------------------------------- helpers
template <class T> struct is_fp { static const bool value = false; };
template <> struct is_fp<float> { static const bool value = true; };
template <> struct is_fp<double> { static const bool value = true; };

template <class T> __device__ __forceinline__ T cvt(float v) { return (T)v; }
template <class T> __device__ __forceinline__ T cvt(double v) { return (T)v; }
template <class T> __device__ __forceinline__ T cvt(int v) { return (T)v; }
template <class T> __device__ __forceinline__ T cvt(unsigned v) { return (T)v; }

// convert_int_rtn of a gather index (kernel/Subscript.cpp:549) and the
// interpreter's periodic wrap (interp/InterpGather.hpp:19-44): add n if
// negative, then modulo n.  Indices below -n are undefined in the reference
// (it reads out of bounds); here they wrap fully.
template <class T> __device__ __forceinline__ long long gather_index(T v, long long n)
{
    long long i;
    if (sizeof(T) == 4 && is_fp<T>::value) i = (long long)floorf((float)v);
    else if (is_fp<T>::value) i = (long long)floor((double)v);
    else i = (long long)v;
    if (i < 0) i += n;
    if (i >= n) i -= n;
    if ((unsigned long long)i >= (unsigned long long)n) {   // far outside [-n, 2n)
        i %= n;
        if (i < 0) i += n;
    }
    return i;
}

// --------------------------------------------------------- unary (1 arg)
template <int OP, class T> __device__ __forceinline__ T f1(T a);

#define CHAI_F1(OP, EXPR) \
    template <> __device__ __forceinline__ float f1<OP, float>(float a) { return EXPR; } \
    template <> __device__ __forceinline__ double f1<OP, double>(double a) { return EXPR; }
#define CHAI_F1F(OP, FF, FD) \
    template <> __device__ __forceinline__ float f1<OP, float>(float a) { return FF(a); } \
    template <> __device__ __forceinline__ double f1<OP, double>(double a) { return FD(a); }
#define CHAI_F1I(OP, EXPR) \
    template <> __device__ __forceinline__ u32 f1<OP, u32>(u32 a) { return EXPR; } \
    template <> __device__ __forceinline__ i32 f1<OP, i32>(i32 a) { return EXPR; }

// arithmetic / logic
CHAI_F1(10, -a)
CHAI_F1I(10, (decltype(a))(0 - a))
CHAI_F1I(15, ~a)
CHAI_F1I(16, (decltype(a))(!a))
CHAI_F1(16, (decltype(a))(!a))
// math (200-266)
CHAI_F1F(200, acosf, acos)
CHAI_F1F(201, acoshf, acosh)
CHAI_F1(202, (decltype(a))(acos(a) / CHAI_PI))
CHAI_F1F(203, asinf, asin)
CHAI_F1F(204, asinhf, asinh)
CHAI_F1(205, (decltype(a))(asin(a) / CHAI_PI))
CHAI_F1F(206, atanf, atan)
CHAI_F1F(208, atanhf, atanh)
CHAI_F1(209, (decltype(a))(atan(a) / CHAI_PI))
CHAI_F1F(211, cbrtf, cbrt)
CHAI_F1F(212, ceilf, ceil)
CHAI_F1F(214, cosf, cos)
CHAI_F1F(215, coshf, cosh)
CHAI_F1F(216, cospif, cospi)
CHAI_F1F(217, erfcf, erfc)
CHAI_F1F(218, erff, erf)
CHAI_F1F(219, expf, exp)
CHAI_F1F(220, exp2f, exp2)
CHAI_F1F(221, exp10f, exp10)
CHAI_F1F(222, expm1f, expm1)
CHAI_F1F(223, fabsf, fabs)
CHAI_F1F(225, floorf, floor)
CHAI_F1(233, (decltype(a))ilogb(a))
CHAI_F1F(235, lgammaf, lgamma)
CHAI_F1F(237, logf, log)
CHAI_F1F(238, log2f, log2)
CHAI_F1F(239, log10f, log10)
CHAI_F1F(240, log1pf, log1p)
CHAI_F1F(241, logbf, logb)
CHAI_F1(246, (decltype(a))__int_as_float(0x7fc00000))
CHAI_F1F(253, rintf, rint)
CHAI_F1F(255, roundf, round)
CHAI_F1F(256, rsqrtf, rsqrt)
CHAI_F1F(257, sinf, sin)
CHAI_F1F(259, sinhf, sinh)
CHAI_F1F(260, sinpif, sinpi)
CHAI_F1F(261, sqrtf, sqrt)
CHAI_F1F(262, tanf, tan)
CHAI_F1F(263, tanhf, tanh)
CHAI_F1(264, (decltype(a))(tan(a * CHAI_PI)))
CHAI_F1F(265, tgammaf, tgamma)
CHAI_F1F(266, truncf, trunc)
// common (300-308)
CHAI_F1(301, (decltype(a))(a * (180.0 / CHAI_PI)))
CHAI_F1(305, (decltype(a))(a * (CHAI_PI / 180.0)))
CHAI_F1(308, (decltype(a))(a > 0 ? 1 : (a < 0 ? -1 : 0)))
// integer (400-415)
CHAI_F1I(400, (decltype(a))(a < 0 ? (decltype(a))(0 - a) : a))
CHAI_F1(400, (decltype(a))fabs(a))
CHAI_F1I(404, (decltype(a))__clz((int)a))
// relational (507-513)
CHAI_F1(507, (decltype(a))(isfinite(a) ? 1 : 0))
CHAI_F1(508, (decltype(a))(isinf(a) ? 1 : 0))
CHAI_F1(509, (decltype(a))(isnan(a) ? 1 : 0))
CHAI_F1(510, (decltype(a))((isfinite(a) && a != 0 && fabs((double)a) >= (sizeof(a) == 4 ? 1.17549435e-38 : 2.2250738585072014e-308)) ? 1 : 0))
CHAI_F1(513, (decltype(a))(signbit(a) ? 1 : 0))

// -------------------------------------------------------- binary (2 args)
template <int OP, class T> __device__ __forceinline__ T f2(T a, T b);

#define CHAI_F2ALL(OP, EXPR) \
    template <> __device__ __forceinline__ float f2<OP, float>(float a, float b) { return EXPR; } \
    template <> __device__ __forceinline__ double f2<OP, double>(double a, double b) { return EXPR; } \
    template <> __device__ __forceinline__ u32 f2<OP, u32>(u32 a, u32 b) { return EXPR; } \
    template <> __device__ __forceinline__ i32 f2<OP, i32>(i32 a, i32 b) { return EXPR; }
#define CHAI_F2FP(OP, EXPR) \
    template <> __device__ __forceinline__ float f2<OP, float>(float a, float b) { return EXPR; } \
    template <> __device__ __forceinline__ double f2<OP, double>(double a, double b) { return EXPR; }
#define CHAI_F2INT(OP, EXPR) \
    template <> __device__ __forceinline__ u32 f2<OP, u32>(u32 a, u32 b) { return EXPR; } \
    template <> __device__ __forceinline__ i32 f2<OP, i32>(i32 a, i32 b) { return EXPR; }

// Packed f32 pairs: the element kernels hold 4 consecutive elements per
// thread; add / sub of f32 operands run as two sm_100 f32x2 instructions
// (round to nearest even per lane, the same IEEE results as the scalar ops,
// half the instruction issue).  The translator never emits the packed
// multiply: ptxas contracts mul.rn.f32x2 followed by add / sub.rn.f32x2 into a
// single-rounding packed FMA.
template <int OP> struct pk2;
template <> struct pk2<11> { static __device__ __forceinline__ unsigned long long op(unsigned long long a, unsigned long long b)
    { unsigned long long d; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; } };
template <> struct pk2<13> { static __device__ __forceinline__ unsigned long long op(unsigned long long a, unsigned long long b)
    { unsigned long long d; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; } };
template <> struct pk2<14> { static __device__ __forceinline__ unsigned long long op(unsigned long long a, unsigned long long b)
    { unsigned long long d; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; } };

template <int OP> __device__ __forceinline__ void f2x4(const float* a, const float* b, float* o)
{
#pragma unroll
    for (int h = 0; h < 2; h++) {
        unsigned long long pa, pb, d;
        asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a[2 * h]), "f"(a[2 * h + 1]));
        asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b[2 * h]), "f"(b[2 * h + 1]));
        d = pk2<OP>::op(pa, pb);
        asm("mov.b64 {%0, %1}, %2;" : "=f"(o[2 * h]), "=f"(o[2 * h + 1]) : "l"(d));
    }
}

CHAI_F2ALL(11, a + b)
CHAI_F2ALL(13, a * b)
CHAI_F2ALL(14, a - b)
CHAI_F2FP(12, a / b)
CHAI_F2INT(12, (decltype(a))(b == 0 ? 0 : a / b))
CHAI_F2INT(17, (decltype(a))(b == 0 ? 0 : a % b))
CHAI_F2FP(17, (decltype(a))fmod(a, b))
CHAI_F2INT(18, (decltype(a))(a << (b & 31)))
CHAI_F2INT(19, (decltype(a))(a >> (b & 31)))
CHAI_F2INT(20, a & b)
CHAI_F2INT(21, a | b)
CHAI_F2INT(22, a ^ b)
CHAI_F2ALL(30, (decltype(a))((a && b) ? 1 : 0))
CHAI_F2ALL(31, (decltype(a))((a || b) ? 1 : 0))
CHAI_F2ALL(32, (decltype(a))(a == b ? 1 : 0))
CHAI_F2ALL(33, (decltype(a))(a != b ? 1 : 0))
CHAI_F2ALL(34, (decltype(a))(a >= b ? 1 : 0))
CHAI_F2ALL(35, (decltype(a))(a > b ? 1 : 0))
CHAI_F2ALL(36, (decltype(a))(a <= b ? 1 : 0))
CHAI_F2ALL(37, (decltype(a))(a < b ? 1 : 0))
CHAI_F2FP(207, (decltype(a))atan2(a, b))
CHAI_F2FP(210, (decltype(a))(atan2(a, b) / CHAI_PI))
CHAI_F2FP(213, (decltype(a))copysign(a, b))
CHAI_F2FP(224, (decltype(a))fdim(a, b))
CHAI_F2FP(227, (decltype(a))fmax(a, b))
CHAI_F2FP(228, (decltype(a))fmin(a, b))
CHAI_F2FP(229, (decltype(a))fmod(a, b))
CHAI_F2FP(232, (decltype(a))hypot(a, b))
CHAI_F2FP(234, (decltype(a))ldexp(a, (int)b))
CHAI_F2FP(243, (decltype(a))(fabs(a) > fabs(b) ? a : (fabs(a) < fabs(b) ? b : fmax(a, b))))
CHAI_F2FP(244, (decltype(a))(fabs(a) < fabs(b) ? a : (fabs(a) > fabs(b) ? b : fmin(a, b))))
CHAI_F2FP(247, (decltype(a))nextafter(a, b))
CHAI_F2FP(248, (decltype(a))pow(a, b))
CHAI_F2FP(249, (decltype(a))pow(a, (decltype(a))(int)b))
CHAI_F2FP(250, (decltype(a))pow(a, b))
CHAI_F2FP(251, (decltype(a))remainder(a, b))
CHAI_F2FP(254, (decltype(a))pow(a, (decltype(a))1 / (decltype(a))(int)b))
CHAI_F2ALL(302, (a < b ? b : a))
// IEEE maximum that returns NaN when either input is NaN (one instruction);
// used by the translator's max-of-affine rewrite where NaN is tested for
__device__ __forceinline__ float max_nan(float a, float b)
{
    float d;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
CHAI_F2ALL(303, (a < b ? a : b))
CHAI_F2FP(306, (decltype(a))(b < a ? 0 : 1))
CHAI_F2INT(401, (decltype(a))(a < b ? b - a : a - b))
template <> __device__ __forceinline__ u32 f2<402, u32>(u32 a, u32 b)
{ unsigned long long c = (unsigned long long)a + b; return c <= 0xffffffffull ? (u32)c : 0xffffffffu; }
template <> __device__ __forceinline__ i32 f2<402, i32>(i32 a, i32 b)
{ long long c = (long long)a + b; return c <= 2147483647ll ? (c >= -2147483647ll - 1 ? (i32)c : (i32)(-2147483647 - 1)) : 2147483647; }
CHAI_F2INT(405, (decltype(a))(((long long)a + (long long)b) >> 1))
CHAI_F2INT(411, (decltype(a))((a & 0x00ffffff) * (b & 0x00ffffff)))
template <> __device__ __forceinline__ u32 f2<412, u32>(u32 a, u32 b) { return __umulhi(a, b); }
template <> __device__ __forceinline__ i32 f2<412, i32>(i32 a, i32 b) { return __mulhi(a, b); }
CHAI_F2INT(413, (decltype(a))(((long long)a + (long long)b + 1) >> 1))
template <> __device__ __forceinline__ u32 f2<414, u32>(u32 a, u32 b) { return __funnelshift_l(a, a, b); }
template <> __device__ __forceinline__ i32 f2<414, i32>(i32 a, i32 b)
{ return (i32)__funnelshift_l((u32)a, (u32)a, (u32)b); }
template <> __device__ __forceinline__ u32 f2<415, u32>(u32 a, u32 b) { return a > b ? a - b : 0u; }
template <> __device__ __forceinline__ i32 f2<415, i32>(i32 a, i32 b)
{ long long c = (long long)a - b; return c > 2147483647ll ? 2147483647 : (c < -2147483648ll ? (i32)(-2147483647 - 1) : (i32)c); }
CHAI_F2ALL(500, (decltype(a))(a == b ? 1 : 0))
CHAI_F2ALL(501, (decltype(a))(a != b ? 1 : 0))
CHAI_F2ALL(502, (decltype(a))(a > b ? 1 : 0))
CHAI_F2ALL(503, (decltype(a))(a >= b ? 1 : 0))
CHAI_F2ALL(504, (decltype(a))(a < b ? 1 : 0))
CHAI_F2ALL(505, (decltype(a))(a <= b ? 1 : 0))
CHAI_F2FP(506, (decltype(a))((a < b || a > b) ? 1 : 0))
CHAI_F2FP(511, (decltype(a))((!isnan(a) && !isnan(b)) ? 1 : 0))
CHAI_F2FP(512, (decltype(a))((isnan(a) || isnan(b)) ? 1 : 0))

// ------------------------------------------------------- ternary (3 args)
template <int OP, class T> __device__ __forceinline__ T f3(T a, T b, T c);

#define CHAI_F3FP(OP, EXPR) \
    template <> __device__ __forceinline__ float f3<OP, float>(float a, float b, float c) { return EXPR; } \
    template <> __device__ __forceinline__ double f3<OP, double>(double a, double b, double c) { return EXPR; }
#define CHAI_F3ALL(OP, EXPR) \
    CHAI_F3FP(OP, EXPR) \
    template <> __device__ __forceinline__ u32 f3<OP, u32>(u32 a, u32 b, u32 c) { return EXPR; } \
    template <> __device__ __forceinline__ i32 f3<OP, i32>(i32 a, i32 b, i32 c) { return EXPR; }

// cond(pred, a, b) (api/chai.h:313-337): pred != 0 ? a : b
CHAI_F3ALL(23, (a != 0 ? b : c))
CHAI_F3FP(226, (decltype(a))fma(a, b, c))
CHAI_F3FP(242, (decltype(a))(a * b + c))
CHAI_F3ALL(300, (a < b ? b : (c < a ? c : a)))
CHAI_F3FP(304, (decltype(a))(a + (b - a) * c))
CHAI_F3FP(307, ([&]() { decltype(a) t = (c - a) / (b - a); t = t < 0 ? 0 : (t > 1 ? 1 : t);
                        return (decltype(a))(t * t * (3 - 2 * t)); }()))
template <> __device__ __forceinline__ u32 f3<406, u32>(u32 a, u32 b, u32 c) { return (a & 0xffffff) * (b & 0xffffff) + c; }
template <> __device__ __forceinline__ i32 f3<406, i32>(i32 a, i32 b, i32 c) { return (a & 0xffffff) * (b & 0xffffff) + c; }
template <> __device__ __forceinline__ u32 f3<407, u32>(u32 a, u32 b, u32 c) { return __umulhi(a, b) + c; }
template <> __device__ __forceinline__ i32 f3<407, i32>(i32 a, i32 b, i32 c) { return __mulhi(a, b) + c; }
template <> __device__ __forceinline__ u32 f3<408, u32>(u32 a, u32 b, u32 c)
{ unsigned long long v = (unsigned long long)a * b + c; return v > 0xffffffffull ? 0xffffffffu : (u32)v; }
template <> __device__ __forceinline__ i32 f3<408, i32>(i32 a, i32 b, i32 c)
{ long long v = (long long)a * b + c; return v > 2147483647ll ? 2147483647 : (v < -2147483648ll ? (i32)(-2147483647 - 1) : (i32)v); }

}  // namespace chai_ops

#endif
