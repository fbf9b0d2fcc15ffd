"""A traced f32 matmul runs on the tcgen05 tensor-core GEMM (GemmPrecision=auto,
the default): the C1 trace (512^3 matmul + sum(C*C), inputs generated in the
trace) and a 4096^3 traced matmul both launch the tensor-core kernel
(chai_cuda_kernel_stats "gemm_tc"), with the split-precision accuracy of the
GEMM parity tests: componentwise-normalised error <= 1e-6 against the FP64
oracle (oracle.gemm_f64 / gemm_entries_f64, the interpreter's matmul in
double, interp/InterpMatmulBase.hpp:50-61).  Thin products (M or N < 32) stay
on the FP32 CUDA-core kernel."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.fixture(scope="module")
def tdev(chai_dev):
    """A context with per-kernel timing on (launch counts per kernel name)."""
    import chai_b200.api as ch
    old = os.environ.get("CHAI_KERNEL_TIMING")
    os.environ["CHAI_KERNEL_TIMING"] = "1"
    try:
        dev = ch.Device()
    finally:
        if old is None:
            del os.environ["CHAI_KERNEL_TIMING"]
        else:
            os.environ["CHAI_KERNEL_TIMING"] = old
    yield dev
    dev.close()


def launches(dev, name):
    ms, n = C.c_double(), C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(dev.ctx, name.encode(), C.byref(ms), C.byref(n), 1), dev.ctx)
    return n.value


def run(ch, dev, inputs, build, out_shape):
    """Record build(*input arrays) over input variables bound to fresh buffers,
    evaluate it on `dev`, return the result."""
    ch._Client.pending, saved = [], ch._Client.pending
    try:
        ins = []
        for arr in inputs:
            H, W = arr.shape
            var = next(ch._Client.vars)
            ins.append((var, ch._Raw([ch._bc(L.BC_VARIABLE, var, 0)], L.F32, W, H)))
        out = build(*[x[1] for x in ins])
        stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    finally:
        ch._Client.pending = saved
    binds = []
    for k, (arr, (var, _)) in enumerate(zip(inputs, ins)):
        bid = 9100 + k
        L.check(L.lib().chai_cuda_buffer_alloc(dev.ctx, bid, arr.nbytes), dev.ctx)
        L.check(L.lib().chai_cuda_upload(dev.ctx, bid, arr.ctypes.data_as(C.c_void_p), arr.nbytes), dev.ctx)
        binds.append((var, L.F32, arr.shape[1], arr.shape[0], 1, 0, bid))
    H, W = out_shape
    binds.append((out.var, L.F32, W, H, 1, 0, 9199))
    dev.evaluate(stmts, binds)
    got = dev.readback(9199, W * H, np.float32).reshape(H, W)
    for b in binds:
        dev.release(b[-1])
    return got


def test_c1_trace_uses_tensor_cores(chai_dev, tdev):
    import bench
    import chai_b200.api as ch
    n = bench.C1_N
    launches(tdev, "gemm_tc")
    s = run(ch, tdev, [], lambda: ch.Arrayf32(bench.c1_expr(ch, ch.RNGf32(ch.RNG_PHILOX, 0))), (1, 1))[0, 0]
    assert launches(tdev, "gemm_tc") >= 1
    A = oracle.rng_fill(n * n, seed=0, limits=(-1.0, 1.0)).reshape(n, n)
    B = oracle.rng_fill(n * n, seed=n * n, limits=(-1.0, 1.0)).reshape(n, n)
    s64 = float((oracle.gemm_f64(A, B) ** 2).sum())
    assert abs(float(s) - s64) <= 1e-5 * s64


def test_4096_traced_matmul_uses_tensor_cores(chai_dev, tdev):
    import chai_b200.api as ch
    n = 4096
    A = oracle.rng_fill(n * n, seed=1, limits=(-1.0, 1.0)).reshape(n, n)
    B = oracle.rng_fill(n * n, seed=2, limits=(-1.0, 1.0)).reshape(n, n)
    launches(tdev, "gemm_tc")
    Cg = run(ch, tdev, [A, B], lambda a, b: ch.Arrayf32(ch.matmul(a, b)), (n, n))
    assert launches(tdev, "gemm_tc") >= 1
    rng = np.random.default_rng(4)
    rows, cols = rng.integers(0, n, 4096), rng.integers(0, n, 4096)
    c64 = oracle.gemm_entries_f64(A, B, rows, cols)
    bound = oracle.gemm_entries_f64(np.abs(A), np.abs(B), rows, cols)
    err = float(np.max(np.abs(Cg[rows, cols].astype(np.float64) - c64) / bound))
    assert err <= 1e-6, err


def test_thin_product_stays_on_cuda_cores(chai_dev, tdev):
    import chai_b200.api as ch
    rng = np.random.default_rng(5)
    A = rng.uniform(-1, 1, (16, 300)).astype(f32)
    B = rng.uniform(-1, 1, (300, 200)).astype(f32)
    launches(tdev, "gemm_tc")
    Cg = run(ch, tdev, [A, B], lambda a, b: ch.Arrayf32(ch.matmul(a, b)), (16, 200))
    assert launches(tdev, "gemm_tc") == 0
    bound = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    assert np.max(np.abs(Cg - oracle.gemm_f64(A, B)) / bound) <= 2.0 ** -18
