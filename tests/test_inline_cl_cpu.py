"""Inline OpenCL kernels (ProgramCL) on the CPU: the recorded statement, the
signature parse (api/ProgramCL.cpp:45-176) and the OpenCL C -> CUDA text that
NVRTC compiles for sm_100a (chai_cuda_trace_source, no device needed)."""
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


def test_image_arguments_are_rejected():
    prog = ch.ProgramCL("__kernel void k(image2d_t img, __global float* a) { }")
    n = 4

    def build():
        a = ch.Arrayf32(ch.zeros_f32(n))
        prog("k", a, a)(n, 1)
        return a
    stmts, kernels, a = record_with_kernels(build)
    st, src = source(stmts, kernels, [(a.var, 4, n, 1, 1, 0, 9)])
    assert st != 0
    assert "image2d_t" in src
