"""Failure detection without a GPU fault: a bounded device wait that runs out
(a barrier nothing arrives on) becomes CHAI_ERR_TIMEOUT on the host and the
context stays usable; host-side injection (CHAI_FAULT_INJECT) makes evaluate
and allocation fail cleanly, and the next call succeeds."""
import ctypes as C
import os
import time

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


def test_bounded_wait_gives_up_and_context_recovers(ch, chai_dev):
    t0 = time.perf_counter()
    st = L.lib().chai_cuda_selftest_wait(chai_dev.ctx, 20.0)
    dt = time.perf_counter() - t0
    assert st == -5                                   # CHAI_ERR_TIMEOUT
    assert 0.015 < dt < 5.0
    # the status word was reset: the next synchronize and a real trace succeed
    L.check(L.lib().chai_cuda_synchronize(chai_dev.ctx), chai_dev.ctx)
    img = oracle.rng_fill(32 * 64, seed=3).reshape(32, 64)
    from tests.test_gpu_trace import kirsch_expr
    assert np.array_equal(ch.Arrayf32(kirsch_expr(ch, ch.make2(img), 64, 32)).read2(), oracle.kirsch(img))


def test_selftest_rejects_bad_limits(chai_dev):
    assert L.lib().chai_cuda_selftest_wait(chai_dev.ctx, 0.0) == -1
    assert L.lib().chai_cuda_selftest_wait(chai_dev.ctx, 5000.0) == -1


@pytest.mark.parametrize("site", ["evaluate", "alloc"])
def test_injected_failures_are_clean(ch, chai_dev, site):
    x = np.arange(64, dtype=np.float32)
    os.environ["CHAI_FAULT_INJECT"] = site
    try:
        with pytest.raises(L.ChaiError) as e:
            ch.Arrayf32(ch.make1(x) * np.float32(2)).read1()
        assert e.value.args and "INJECTED" in str(e.value)
    finally:
        del os.environ["CHAI_FAULT_INJECT"]
    # the same work succeeds once the injection is off
    assert np.array_equal(ch.Arrayf32(ch.make1(x) * np.float32(2)).read1(), x * np.float32(2))


def test_gemm_wait_runs_out_and_next_gemm_is_exact(ch):
    """A bounded wait inside the tcgen05 GEMM runs out: with
    CHAI_FAULT_INJECT=gemm_stall the one-CTA kernel's producer (CTA 0) posts
    one chunk's expected bytes but issues no copy, so the MMA's wait gives up
    after its limit, the kernel drains its MMAs, frees TMEM and returns; the
    host reads CHAI_ERR_TIMEOUT from the status word, and the next GEMM on
    the same context is bit-identical to one before the failure."""
    import torch
    dev = ch.Device(config="GemmPair=0")
    try:
        M, N, K = 512, 384, 256
        g = torch.Generator(device="cuda").manual_seed(5)
        A = torch.rand((M, K), device="cuda", generator=g) * 2 - 1
        B = torch.rand((K, N), device="cuda", generator=g) * 2 - 1

        def gemm():
            Cm = torch.full((M, N), float("nan"), device="cuda")
            d = L.chai_gemm_desc(L.GEMM_BF16X3, 0, 0, 0, M, N, K, A.data_ptr(), K, B.data_ptr(), N, Cm.data_ptr(), N,
                                 1.0, 0.0, 1, 0, 0, 0)
            st = L.lib().chai_cuda_gemm(dev.ctx, C.byref(d))
            return st, Cm
        st, before = gemm()
        assert st == 0
        L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
        os.environ["CHAI_FAULT_INJECT"] = "gemm_stall"
        try:
            t0 = time.perf_counter()
            st, _ = gemm()
            sync = L.lib().chai_cuda_synchronize(dev.ctx)
            dt = time.perf_counter() - t0
        finally:
            del os.environ["CHAI_FAULT_INJECT"]
        assert st == 0 and sync == -5, (st, sync)      # CHAI_ERR_TIMEOUT
        assert 1.0 < dt < 30.0, dt
        st, after = gemm()
        assert st == 0
        L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
        assert torch.equal(before, after) and torch.isfinite(after).all()
    finally:
        dev.close()
