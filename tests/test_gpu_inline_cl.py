"""Inline OpenCL kernels (ProgramCL) on the GPU: the reference sample
(sample/inline_cl.cpp), __local memory with barriers, a 2-D NDRange, an
integer kernel, in-place update of an array from an earlier trace, and replay
from the plan cache.  Expected values are computed with numpy in the same
float32 arithmetic (bit-exact), except the tree reduction (1e-6 relative)."""
import ctypes as C

import numpy as np
import pytest

from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.fixture
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


def test_reference_sample_inline_cl(ch):
    N = 20
    prog = ch.ProgramCL("__kernel void add_scalar(__global float* a, float s)"
                        "{"
                        "  a[get_global_id(0)] += s;"
                        "}")
    cpuA = np.arange(N, dtype=f32)
    cpuB = (N - np.arange(N)).astype(f32)
    A, B = ch.make1(cpuA), ch.make1(cpuB)
    Cv = ch.Arrayf32(A + B)
    prog("add_scalar", Cv, f32(1.5))(N, 1)
    Cv.assign(Cv + (A - f32(3.3)))
    got = Cv.read1()
    want = ((cpuA + cpuB) + f32(1.5)) + (cpuA - f32(3.3))
    assert np.array_equal(got, want)


BLOCK_SUM = """
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
"""


def test_local_memory_block_sum(ch):
    n, wg = 1000, 128
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, n).astype(f32)
    prog = ch.ProgramCL(BLOCK_SUM)
    X = ch.make1(x)
    out = ch.Arrayf32(ch.zeros_f32(8))
    prog("block_sum", X, wg, out, np.uint32(n))(1024, wg)
    got = out.read1()
    want = np.array([x[g * wg:(g + 1) * wg].astype(np.float64).sum() for g in range(8)])
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)


def test_two_dimensional_ndrange_and_work_item_functions(ch):
    W, H = 64, 12
    prog = ch.ProgramCL("""
    __kernel void fill2(__global float* a, uint W)
    {
        const uint x = get_global_id(0), y = get_global_id(1);
        a[y * W + x] = (float)x + 1000.0f * (float)y + (float)get_work_dim() * 0.25f
                       + (float)(get_group_id(1) * get_num_groups(0) + get_group_id(0)) * 1e-3f;
    }""")
    a = ch.Arrayf32(ch.zeros_f32(W, H))
    prog("fill2", a, np.uint32(W))(W, H, 16, 4)
    got = a.read2()
    y, x = np.mgrid[0:H, 0:W].astype(f32)
    gid = ((y // 4) * (W // 16) + (x // 16)).astype(f32)
    want = x + f32(1000) * y + f32(2 * 0.25) + gid * f32(1e-3)
    assert np.array_equal(got, want)


def test_integer_kernel_and_following_trace(ch):
    n = 256
    prog = ch.ProgramCL("""
    __kernel void mix_bits(__global uint* a, uint k)
    {
        const size_t i = get_global_id(0);
        a[i] = (a[i] ^ k) * 2654435761u + (uint)i;
    }""")
    base = np.arange(n, dtype=np.uint32) * np.uint32(7)
    A = ch.Arrayu32(ch.make1(base))
    prog("mix_bits", A, np.uint32(0xdeadbeef))(n, 64)
    B = ch.Arrayu32(A + np.uint32(1))
    got = B.read1()
    with np.errstate(over="ignore"):
        want = ((base ^ np.uint32(0xdeadbeef)) * np.uint32(2654435761) + np.arange(n, dtype=np.uint32)
                + np.uint32(1))
    assert np.array_equal(got, want)


def test_kernel_updates_array_from_earlier_trace(ch):
    n = 96
    x = np.linspace(-1, 1, n).astype(f32)
    A = ch.Arrayf32(ch.make1(x) * f32(2))
    assert np.array_equal(A.read1(), x * f32(2))           # A now lives in HBM
    prog = ch.ProgramCL("__kernel void sq(__global float* a) { size_t i = get_global_id(0); a[i] = a[i] * a[i]; }")
    prog("sq", A)(n, 32)
    got = A.read1()
    assert np.array_equal(got, (x * f32(2)) * (x * f32(2)))


def test_inline_kernel_trace_replays(ch, chai_dev):
    N = 64
    prog = ch.ProgramCL("__kernel void add_scalar(__global float* a, float s) { a[get_global_id(0)] += s; }")
    n0 = C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(chai_dev.ctx, b"plan_replay", None, C.byref(n0), 0), chai_dev.ctx)
    for k in range(3):
        a = np.full(N, k, dtype=f32)
        A = ch.make1(a)
        Cv = ch.Arrayf32(A * f32(2))
        prog("add_scalar", Cv, f32(0.5))(N, 16)
        assert np.array_equal(Cv.read1(), a * f32(2) + f32(0.5))
    n1 = C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(chai_dev.ctx, b"plan_replay", None, C.byref(n1), 0), chai_dev.ctx)
    assert n1.value - n0.value == 2


def test_kernel_arguments_equal_to_other_variables_get_their_own_storage(ch):
    """Two arrays made by the same expression (one node after deduplication)
    stay two arrays when a kernel updates them: each argument, and every
    other variable of that value, keeps its own contents."""
    n = 128
    prog = ch.ProgramCL("""
    __kernel void two(__global float* a, __global float* b) { const size_t i = get_global_id(0); a[i] = 1.0f; b[i] = 2.0f; }
    __kernel void one(__global float* a) { a[get_global_id(0)] = 5.0f; }""")
    A, B = ch.Arrayf32(ch.zeros_f32(n)), ch.Arrayf32(ch.zeros_f32(n))
    prog("two", A, B)(n, 64)
    assert np.array_equal(A.read1(), np.full(n, 1, f32)) and np.array_equal(B.read1(), np.full(n, 2, f32))
    C, D = ch.Arrayf32(ch.zeros_f32(n)), ch.Arrayf32(ch.zeros_f32(n))
    prog("one", C)(n, 64)
    assert np.array_equal(C.read1(), np.full(n, 5, f32)) and np.array_equal(D.read1(), np.zeros(n, f32))
