"""Inline OpenCL kernels (ProgramCL) on the CPU: the recorded statement, the
signature parse (api/ProgramCL.cpp:45-176) and the OpenCL C -> CUDA text that
NVRTC compiles for sm_100a (chai_cuda_trace_source, no device needed): the
scalar language, and vector types, swizzles, conversions, atomics, work-group
copies and image2d_t parameters."""
import ctypes as C

import numpy as np
import pytest

import chai_b200.api as ch
from chai_b200 import _lib as L

f32 = np.float32

ADD_SCALAR = ("__kernel void add_scalar(__global float* a, float s)"
              "{"
              "  a[get_global_id(0)] += s;"
              "}")

BLOCK_SUM = """
// one partial sum per work group, through __local memory
__kernel void block_sum(__global const float* x, __local float* t, __global float* out, uint n)
{
    const uint l = get_local_id(0), g = get_global_id(0);
    t[l] = g < n ? x[g] : 0.0f;
    barrier(CLK_LOCAL_MEM_FENCE);
    for (uint s = get_local_size(0) / 2; s > 0; s >>= 1) {
        if (l < s) t[l] += t[l + s];
        barrier(CLK_LOCAL_MEM_FENCE);
    }
    if (l == 0) out[get_group_id(0)] = t[0];
}
__kernel void unused(__local int* scratch) { }
"""


def record_with_kernels(build):
    ch._Client.pending, ch._Client.kernels = [], []
    keep = build()
    stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    kernels = ch._Client.kernels
    ch._Client.pending, ch._Client.kernels = [], []
    return stmts, kernels, keep


def source(stmts, kernels, binds=()):
    desc, keep = ch.build_desc(stmts, 1, kernels)
    b = (L.chai_buffer_binding * max(1, len(binds)))()
    for i, x in enumerate(binds):
        b[i] = L.chai_buffer_binding(*x)
    buf = C.create_string_buffer(1 << 21)
    need = C.c_size_t()
    st = L.lib().chai_cuda_trace_source(C.byref(desc), b, len(binds), None, buf, len(buf), C.byref(need))
    return st, buf.value.decode()


def test_signature_parse_matches_reference_rules():
    p = ch.ProgramCL(BLOCK_SUM)
    assert p._sigs["block_sum"] == [(L.KARG_ARRAY, L.F32), (L.KARG_LOCAL, L.F32), (L.KARG_ARRAY, L.F32),
                                    (L.KARG_SCALAR, L.U32)]
    assert p._sigs["unused"] == [(L.KARG_LOCAL, L.I32)]
    with pytest.raises(ValueError):
        p("missing")


def test_sample_inline_cl_records_and_compiles():
    """sample/inline_cl.cpp: C = A + B; (prog, "add_scalar", C, 1.5f)(N, 1); C += A - 3.3f."""
    N = 20
    prog = ch.ProgramCL(ADD_SCALAR)

    def build():
        A = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(1), ch._sc(N), ch._op(62)], N, 1, 1))
        B = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=8), ch._sc(1), ch._sc(1), ch._sc(N), ch._op(62)], N, 1, 1))
        Cv = ch.Arrayf32(A + B)
        prog("add_scalar", Cv, f32(1.5))(N, 1)
        Cv.assign(Cv + (A - f32(3.3)))
        return Cv
    stmts, kernels, Cv = record_with_kernels(build)
    assert any(cells[-1][:2] == (L.BC_OPCODE, 50) for _, _, cells in stmts)
    assert kernels[0][1] == "add_scalar" and kernels[0][2][1] == (L.KARG_SCALAR, L.F32, 0, 0, 1.5)
    st, src = source(stmts, kernels, [(Cv.var, 4, N, 1, 1, 0, 9)])
    assert st == 0, src
    # the kernel is a barrier between two element kernels
    assert src.count('extern "C" __global__ void add_scalar') == 1
    assert src.count("chai_group") == 2


def test_local_memory_pointer_is_placed_in_dynamic_shared_memory():
    n, wg = 1000, 128
    prog = ch.ProgramCL(BLOCK_SUM)

    def build():
        x = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(1), ch._sc(n), ch._op(62)], n, 1, 1))
        x = ch.Arrayf32(x)
        out = ch.Arrayf32(ch.zeros_f32(8))
        prog("block_sum", x, wg, out, np.uint32(n))(1024, wg)
        return out
    stmts, kernels, out = record_with_kernels(build)
    st, src = source(stmts, kernels, [(out.var, 4, 8, 1, 1, 0, 9)])
    assert st == 0, src
    assert "extern __shared__ __align__(16) unsigned char chai_cl_lmem[]; t = reinterpret_cast<float*>(chai_cl_lmem + 0);" in src
    assert "__shared__" not in src.split("void unused")[1].split("{")[0]   # parameter qualifier removed
    import re
    assert not re.search(r"\b__global\b(?!_)", src.split("// ---- program text")[1])


def compile_call(text, name, arrays, extra=()):
    """Record `prog(name, *arrays, *extra)(64, 16)` over the given
    (precision, W, H) arrays and compile the trace; (status, source)."""
    prog = ch.ProgramCL(text)
    zeros = {L.F32: ch.zeros_f32, L.F64: ch.zeros_f64, L.I32: ch.zeros_i32, L.U32: ch.zeros_u32}

    def build():
        arrs = [ch._ARR[p](zeros[p](w, h)) for p, w, h in arrays]
        prog(name, *arrs, *extra)(64, 16)
        return arrs
    stmts, kernels, arrs = record_with_kernels(build)
    return source(stmts, kernels)


VEC_OPS = """
__kernel void vec_ops(__global float* a, __global float* out, __global int* iout, uint n)
{
    const size_t i = get_global_id(0);
    if (i >= n) return;
    float4 v = vload4(i, a);
    float4 w = (float4)(1.0f, 2.0f, 3.0f, 4.0f);
    float4 u = v * w + (float4)(0.5f);
    u.xy = u.yx;
    u.zw += (float2)(1.0f, -1.0f);
    u.s0 = u.s3 * 2.0f;
    float2 lo = u.lo, hi = u.hi;
    float4 m = mix(u, w, 0.25f);
    m = clamp(m, -4.0f, 4.0f);
    m = fmax(m, fmin(u, w));
    int4 c = u > w;
    float4 s = select(u, w, c);
    float d = dot(s.xyz, w.xyz) + length(hi) + distance(lo, hi);
    float3 cr = cross(s.xyz, w.xyz);
    float4 nrm = normalize(m);
    int4 iv = convert_int4_sat_rte(m * 1000.0f);
    uint4 bits = as_uint4(nrm);
    vstore4(sqrt(fabs(nrm)) + exp(-fabs(m)) + sin(s) + (float4)(d, cr), i, out);
    iout[i] = iv.x + iv.y + iv.z + iv.w + (int)(bits.x & 1u) + any(c) + all(c) + popcount(iv.x) + clz(iv.y);
}
"""

DVEC_WIDE = """
#pragma OPENCL EXTENSION cl_khr_fp64 : enable
__kernel void dvec(__global double* a, __global long* b, uint n)
{
    const size_t i = get_global_id(0);
    double2 v = vload2(i, a);
    long2 l = convert_long2(v * 10.0);
    v.even = v.odd;
    b[i] = l.x + l.y + (long)as_ulong(v.x) + add_sat(l.x, l.y) + mul_hi(l.x, l.y);
    vstore2(v + convert_double2(l), i, a);
}
__kernel void wide(__global float* a, __global uint* u)
{
    const size_t i = get_global_id(0);
    float8 v = vload8(i, a);
    float16 w = (float16)(v, v.s76543210);
    uint16 k = convert_uint16_sat(w);
    v.lo = v.hi * 2.0f;
    v.s0123 = v.s4567 + 1.0f;
    w.odd = w.even;
    vstore8(v + w.lo + w.hi, i, a);
    u[i] = k.sF + k.s0 + rotate(k.s1, 3u) + hadd(k.s2, k.s3);
}
"""

ATOMS = """
__kernel void hist(__global const uint* x, __global uint* h, __local uint* lh, uint n, uint bins)
{
    const uint l = get_local_id(0);
    for (uint b = l; b < bins; b += get_local_size(0)) lh[b] = 0;
    barrier(CLK_LOCAL_MEM_FENCE);
    const size_t g = get_global_id(0);
    if (g < n) atomic_inc(&lh[x[g] % bins]);
    barrier(CLK_LOCAL_MEM_FENCE);
    for (uint b = l; b < bins; b += get_local_size(0)) atomic_add(&h[b], lh[b]);
}
__kernel void tile_rev(__global const float4* src, __global float4* dst, __local float4* t)
{
    event_t e = async_work_group_copy(t, src + get_group_id(0) * get_local_size(0), get_local_size(0), 0);
    wait_group_events(1, &e);
    const uint l = get_local_id(0);
    dst[get_global_id(0)] = t[get_local_size(0) - 1 - l].wzyx;
}
__kernel void atoms(__global int* a, __global ulong* b, __global float* f)
{
    atomic_max(&a[0], (int)get_global_id(0));
    atomic_min(&a[1], -(int)get_global_id(0));
    atomic_cmpxchg(&a[2], 0, 1);
    atomic_xchg(&a[3], 7);
    atomic_or(&a[4], 1 << (get_global_id(0) & 31));
    atom_add(&b[0], (ulong)get_global_id(0));
    atomic_add(&f[0], 1.0f);
    atomic_sub(&a[5], 2);
    atomic_dec(&a[6]);
}
"""

IMAGES = """
__constant sampler_t smp = CLK_NORMALIZED_COORDS_FALSE | CLK_ADDRESS_CLAMP | CLK_FILTER_NEAREST;
const sampler_t lin = CLK_NORMALIZED_COORDS_TRUE | CLK_ADDRESS_REPEAT | CLK_FILTER_LINEAR;
__kernel void img(__read_only image2d_t src, __global float* out, __write_only image2d_t dst)
{
    const int x = get_global_id(0), y = get_global_id(1);
    float4 p = read_imagef(src, smp, (int2)(x - 1, y)) + read_imagef(src, smp, (int2)(x + 1, y));
    float2 uv = (float2)((x + 0.5f) / get_image_width(src), (y + 0.5f) / get_image_height(src));
    p += read_imagef(src, lin, uv);
    vstore4(p, y * get_image_width(src) + x, out);
    write_imagef(dst, (int2)(x, y), p * 0.5f);
}
__kernel void dimg(read_only image2d_t src, __global double* out)
{
    const int x = get_global_id(0), y = get_global_id(1);
    double2 v = as_double2(read_imageui(src, smp, (int2)(x, y)));
    vstore2(v, y * get_image_width(src) + x, out);
}
"""


@pytest.mark.parametrize("text,name,arrays,extra", [
    (VEC_OPS, "vec_ops", [(L.F32, 256, 1), (L.F32, 256, 1), (L.I32, 64, 1)], (np.uint32(64),)),
    (DVEC_WIDE, "dvec", [(L.F64, 128, 1), (L.F64, 64, 1)], (np.uint32(64),)),
    (ATOMS, "hist", [(L.U32, 64, 1), (L.U32, 64, 1)], (64, np.uint32(64), np.uint32(64))),
    (IMAGES, "img", [(L.F32, 32, 16), (L.F32, 512, 1), (L.F32, 32, 16)], ()),
])
def test_vector_image_and_atomic_programs_compile(text, name, arrays, extra):
    st, src = compile_call(text, name, arrays, extra)
    assert st == 0, src[-3000:]
    body = src.split("// ---- program text")[-1]
    assert "chai_cl::vec<" in body
    assert "float4" not in body.replace("chai_cl::vec<float, 4>", "")


def test_vector_rewrites():
    st, src = compile_call(VEC_OPS, "vec_ops", [(L.F32, 256, 1), (L.F32, 256, 1), (L.I32, 64, 1)],
                           (np.uint32(64),))
    assert st == 0
    body = src.split("// ---- program text")[-1]
    # literals, assigned and read swizzles, conversions and reinterpretations
    assert "chai_cl::make<chai_cl::vec<float, 4>>(1.0f, 2.0f, 3.0f, 4.0f)" in body
    assert "u.chai_swl<0,1>() = u.chai_swr<1,0>();" in body
    assert "u.chai_swl<2,3>() += chai_cl::make<chai_cl::vec<float, 2>>(1.0f, -1.0f);" in body
    assert "u.chai_sw1<0>() = u.chai_sw1<3>() * 2.0f;" in body
    assert "u.chai_lo(), hi = u.chai_hi();" in body
    assert "chai_cl::convert<int, 4, 1, 1>(m * 1000.0f)" in body
    assert "chai_cl::as_type<chai_cl::vec<unsigned int, 4>>(nrm)" in body
    # single x / y / z / w components stay members
    assert "iv.x + iv.y + iv.z + iv.w" in body
    st, src = compile_call(DVEC_WIDE, "wide", [(L.F32, 512, 1), (L.U32, 64, 1)])
    assert st == 0
    body = src.split("// ---- program text")[-1]
    assert "w.chai_odd_l() = w.chai_even();" in body
    assert "v.chai_swl<0,1,2,3>() = v.chai_swr<4,5,6,7>() + 1.0f;" in body
    assert "k.chai_sw1<15>() + k.chai_sw1<0>()" in body


def test_member_names_in_vector_free_programs_are_left_alone():
    text = """
    typedef struct { float lo, hi, sa; } range;
    __kernel void spans(__global float* a)
    {
        range r; r.lo = a[0]; r.hi = a[1]; r.sa = r.hi - r.lo;
        a[get_global_id(0)] = r.sa;
    }"""
    st, src = compile_call(text, "spans", [(L.F32, 64, 1)])
    assert st == 0, src[-2000:]
    assert "r.lo = a[0]; r.hi = a[1]; r.sa = r.hi - r.lo;" in src


def test_image_parameters():
    st, src = compile_call(IMAGES, "img", [(L.F32, 32, 16), (L.F32, 512, 1), (L.F32, 32, 16)])
    assert st == 0, src[-2000:]
    body = src.split("// ---- program text")[-1]
    # pointer + packed extent per image, rebuilt at the top of the body
    assert "unsigned char* chai_img_src, long long chai_imgd_src" in body
    assert "const chai_cl::image2d src = {chai_img_src," in body
    assert "read_only" not in body and "write_only" not in body
    # an f64 array: 2 values per texel
    st, src = compile_call(IMAGES, "dimg", [(L.F64, 16, 4), (L.F64, 64, 1)])
    assert st == 0, src[-2000:]
    # rows must be whole 16-byte texels: 6 floats are not
    st, src = compile_call(IMAGES, "img", [(L.F32, 6, 4), (L.F32, 512, 1), (L.F32, 32, 16)])
    assert st != 0 and "16-byte texels" in src
    for bad, word in (("__kernel void k(image3d_t v, __global float* a) { }", "image3d_t"),
                      ("__kernel void k(sampler_t s, __global float* a) { }", "sampler_t")):
        prog = ch.ProgramCL(bad)
        n = 4

        def build():
            a = ch.Arrayf32(ch.zeros_f32(n))
            prog("k", 0, a)(n, 1)       # neither parameter kind is an array one
            return a
        stmts, kernels, a = record_with_kernels(build)
        st, src = source(stmts, kernels)
        assert st != 0 and word in src


def test_local_memory_is_sized_by_the_declared_element_type():
    prog = ch.ProgramCL(ATOMS)
    assert prog._vbytes["tile_rev"] == [16, 16, 16]
    assert prog._vbytes["hist"] == [0, 0, 0, 0, 0]
    st, src = compile_call(ATOMS, "tile_rev", [(L.F32, 256, 1), (L.F32, 256, 1)], (16,))
    assert st == 0, src[-2000:]
    assert "t = reinterpret_cast<chai_cl::vec<float, 4>*>(chai_cl_lmem + 0);" in src

    def build():
        a = ch.Arrayf32(ch.zeros_f32(256))
        prog("tile_rev", a, a, 16)(64, 16)
        return a
    _, kernels, _ = record_with_kernels(build)
    assert kernels[0][2][2] == (L.KARG_LOCAL, L.F32, 0, 0, 16.0)     # 16 float4: sized by the declared type


def test_vector_scalar_arguments_are_rejected():
    prog = ch.ProgramCL("__kernel void k(__global float* a, float4 v) { }")
    a = ch.Arrayf32(ch.zeros_f32(4))
    with pytest.raises(TypeError):
        prog("k", a, 1.0)(4, 1)


def test_local_offsets_follow_the_declared_element_sizes():
    text = """
    typedef struct { float a, b, c; } trip;
    __kernel void k(__local long* a, __local float4* b, __local uchar* c, __global float* out) { }
    __kernel void s(__local trip* t, __global float* out) { }"""
    prog = ch.ProgramCL(text)

    def build():
        out = ch.Arrayf32(ch.zeros_f32(64))
        prog("k", 3, 2, 5, out)(64, 16)
        return out
    stmts, kernels, _ = record_with_kernels(build)
    st, src = source(stmts, kernels)
    assert st == 0, src[-2000:]
    # 3 longs = 24 B -> 32; 2 float4 = 32 B; 5 uchars
    assert "a = reinterpret_cast<long*>(chai_cl_lmem + 0);" in src
    assert "b = reinterpret_cast<chai_cl::vec<float, 4>*>(chai_cl_lmem + 32);" in src
    assert "c = reinterpret_cast<uchar*>(chai_cl_lmem + 64);" in src

    def build_s():
        out = ch.Arrayf32(ch.zeros_f32(64))
        prog("s", 4, out)(64, 16)
        return out
    stmts, kernels, _ = record_with_kernels(build_s)
    st, src = source(stmts, kernels)
    assert st != 0 and "unknown size" in src


def test_vector_rewrite_edge_cases_compile():
    """Swizzles through '->' and on array elements, upper-case hex
    components, scalar convert_ / as_ names, a literal as a call argument,
    vector compound assignment and comparisons feeding select()."""
    text = """
    typedef struct { float4 p; int n; } item;
    __kernel void edge(__global item* it, __global float* out, __global uint* u)
    {
        const size_t i = get_global_id(0);
        __global item* q = it + i;
        float4 v = q->p;
        q->p.xy = v.zw;
        float2 w = (&it[i])->p.SAB;
        v *= (float4)(2.0f);
        v.hi -= w;
        int4 m = isgreater(v, (float4)(0.0f)) & (v != v.wzyx);
        u[i] = as_uint(out[i]) ^ convert_uint_sat(-1.5f) ^ (uint)convert_int_rtn(v.x);
        out[i] = dot(select((float4)(0.0f), v, m), (float4)(1.0f, 0.5f, 0.25f, 0.125f));
    }"""
    st, src = compile_call(text, "edge", [(L.F32, 256, 1), (L.F32, 64, 1), (L.U32, 64, 1)])
    assert st == 0, src[-3000:]
    body = src.split("// ---- program text")[-1]
    assert "q->p.chai_swl<0,1>() = v.chai_swr<2,3>();" in body
    assert "->p.chai_swr<10,11>();" in body
    assert "v.chai_hi_l() -= w;" in body
    assert "chai_cl::as_type<unsigned int>(out[i])" in body and "chai_cl::convert<unsigned int, 1, 1, 0>(-1.5f)" in body


def test_attributes_between_kernel_and_void():
    """`__kernel __attribute__((...)) void name(...)`: the reference's parser
    skips every token up to `void` (api/ProgramCL.cpp:156-177); the attribute
    is dropped from the CUDA text."""
    text = """
    __kernel __attribute__((reqd_work_group_size(64, 1, 1))) void scale(__global float* a, float s)
    { a[get_global_id(0)] *= s; }"""
    prog = ch.ProgramCL(text)
    assert prog._sigs["scale"] == [(L.KARG_ARRAY, L.F32), (L.KARG_SCALAR, L.F32)]
    st, src = compile_call(text, "scale", [(L.F32, 64, 1)], (f32(2.0),))
    assert st == 0, src[-2000:]
    assert "__attribute__" not in src.split("// ---- program text")[-1]
    assert 'extern "C" __global__ void scale(' in src


def test_half_storage_functions_compile():
    """vload_half* / vstore_half* (all rounding modes, aligned forms, float
    and double sources) over `half` storage."""
    text = """
    __kernel void halves(__global const float* x, __global half* h, __global float* back,
                         __global const double* d, __global half* hd)
    {
        const size_t i = get_global_id(0);
        vstore_half(x[i], i, h);
        vstore_half_rtz(x[i], i + 64, h);
        back[i] = vload_half(i, h) + vload_half(i + 64, h);
        float4 v = vload4(0, x);
        vstore_half4_rtp(v, 40, h);
        vstorea_half3(v.xyz, 20, h);
        float3 w = vloada_half3(20, h);
        float8 z = vload_half8(2, h);
        vstore_half8_rtn(z, 3, h);
        vstore_half_rte(d[i], i, hd);
        back[i + 64] = w.x + z.s7 + vload_half2(1, hd).y;
    }"""
    st, src = compile_call(text, "halves", [(L.F32, 64, 1), (L.U32, 128, 1), (L.F32, 128, 1), (L.F64, 64, 1),
                                            (L.U32, 64, 1)])
    assert st == 0, src[-3000:]


def test_kernel_head_parser_edge_cases():
    """Kernel heads as api/ProgramCL.cpp:145-177 finds them: `kernel` or
    `__kernel`, attributes before `void`, several kernels, and words such as
    "kernel" in comments or identifiers that head nothing."""
    text = """
    // this kernel computes nothing; my_kernel is not a kernel head
    int my_kernel_helper(int x) { return x; }
    kernel void a(global float* x) { }
    __kernel __attribute__((vec_type_hint(float4))) __attribute__((reqd_work_group_size(8, 8, 1)))
    void b(__global uint* y, __local float2* t, float s) { }
    """
    heads = ch._cl_kernel_heads(text)
    assert [h[0] for h in heads] == ["a", "b"]
    p = ch.ProgramCL(text)
    assert p._sigs["a"] == [(L.KARG_ARRAY, L.F32)]
    # float2 is no scalar keyword of the reference's parser: no precision
    assert p._sigs["b"] == [(L.KARG_ARRAY, L.U32), (L.KARG_LOCAL, -1), (L.KARG_SCALAR, L.F32)]
    assert p._vbytes["b"] == [0, 8, 0]
