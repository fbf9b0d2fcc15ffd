"""The allocation-free reduction entry point (chai_cuda_reduce_noalloc)
against the regular one (chai_cuda_reduce), through the C ABI.

It serves callers that must not allocate device memory when they reduce; its
partial sums live in a fixed device array shared by every call.  Two calls in
a row must both agree with the regular entry point (the second call reuses
the array the first one filled).  Results agree within 1e-12 relative: both
accumulate in FP64, the two launches may split the array into a different
number of blocks, so the summation order can differ.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_noalloc_reduce_matches_regular_entry_point(chai_dev):
    import torch
    lib = L.lib()
    rng = np.random.default_rng(11)
    cases = [(0, 1 << 20, 1), (1, 1000003, 1), (2, 1 << 18, 1), (0, 4096, 7)]
    for op, n, slots in cases:
        a = torch.from_numpy(rng.standard_normal(n * slots).astype(np.float32)).cuda()
        b = torch.from_numpy(rng.standard_normal(n * slots).astype(np.float32)).cuda()
        want = (C.c_double * slots)()
        L.check(lib.chai_cuda_reduce(chai_dev.ctx, op, 4, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                     n, slots, want), chai_dev.ctx)
        out = torch.empty(slots, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()
        for call in range(2):
            out.fill_(float("nan"))
            st = lib.chai_cuda_reduce_noalloc(op, 4, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), n, slots,
                                              C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
            assert st == 0, (op, n, slots, call, st)
            got = out.cpu().numpy()
            assert np.allclose(got, np.frombuffer(want, dtype=np.float64), rtol=1e-12, atol=1e-12 * n), \
                (op, n, slots, call, got, list(want))


def test_noalloc_reduce_rejects_too_many_slots(chai_dev):
    import torch
    a = torch.zeros(8193, dtype=torch.float32, device="cuda")
    out = torch.zeros(8193, dtype=torch.float64, device="cuda")
    st = L.lib().chai_cuda_reduce_noalloc(0, 4, C.c_void_p(a.data_ptr()), None, 1, 8193, C.c_void_p(out.data_ptr()),
                                          None)
    assert st == -2
