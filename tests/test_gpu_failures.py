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
