"""The allocation-free reduction entry point (chai_cuda_reduce_noalloc),
through the C ABI.

It serves callers that must not allocate device memory when they reduce (a
pre-sized arena owns the GPU, or an allocation could block or fail late); its
partial sums live in one fixed device array that every call shares.  Each
case runs two calls in a row (the second reuses the array the first one
filled) and checks both against the oracle -- the reference interpreter's
double accumulation (oracle.sum_f32 / oracle.dot_f32 for f32,
interp/InterpAccum.cpp:13-70 and interp/InterpDotprod.cpp:14-60 restated as
an FP64 numpy sum for f64, i32 and u32) -- and against the regular entry
point chai_cuda_reduce.

Tolerances: integer arrays are summed exactly (every partial and total is an
integer below 2^53), so i32 / u32 sums and dot products must be equal; f32 /
f64 results and integer means (the sum times 1/n here, the sum divided by n
in the interpreter) agree within 1e-13 of the sum of magnitudes (both sides
accumulate in FP64 in different orders).

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu

def make(prec, count, rng):
    if prec == L.F32:
        return rng.standard_normal(count).astype(np.float32)
    if prec == L.F64:
        return rng.standard_normal(count)
    if prec == L.I32:
        return rng.integers(-30000, 30000, count, dtype=np.int32)
    return rng.integers(0, 1 << 32, count, dtype=np.uint64).astype(np.uint32)


def oracle_reduce(op, prec, a, b, n, slots):
    """FP64 sum / mean / dot of each slot, as the interpreter accumulates."""
    out, mag = [], []
    for s in range(slots):
        x = a[s * n:(s + 1) * n]
        if op == 2:
            y = b[s * n:(s + 1) * n]
            if prec == L.F32:
                v = oracle.dot_f32(x, y)
            else:
                # the element product is taken in the array type (u32 wraps), then summed in double
                p = x * y
                v = float(np.sum(p.astype(np.float64)))
            m = float(np.sum(np.abs(x.astype(np.float64) * y.astype(np.float64))))
        else:
            v = oracle.sum_f32(x) if prec == L.F32 else float(np.sum(x.astype(np.float64)))
            m = float(np.sum(np.abs(x.astype(np.float64))))
        if op == 1:
            v = v / n if n else float("nan")
            m = m / n if n else 0.0
        out.append(v)
        mag.append(m)
    return np.array(out), np.array(mag)


def regular(dev, op, prec, a, b, n, slots):
    want = (C.c_double * slots)()
    L.check(L.lib().chai_cuda_reduce(dev.ctx, op, prec, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                     n, slots, want), dev.ctx)
    return np.frombuffer(want, dtype=np.float64).copy()


def agree(op, prec, got, want, mag):
    if prec in (L.I32, L.U32) and op != 1:
        return np.array_equal(got, want, equal_nan=True)
    # floating point, and integer means (the sum times 1/n against the sum / n)
    return np.allclose(got, want, rtol=0, atol=0, equal_nan=True) or \
        bool(np.all((np.abs(got - want) <= 1e-13 * mag) | (np.isnan(got) & np.isnan(want))))


CASES = [
    # (op, prec, n, slots)
    (0, L.F32, 1 << 20, 1), (1, L.F32, 1000003, 1), (2, L.F32, 1 << 18, 1), (0, L.F32, 4096, 7),
    (0, L.F64, 1 << 20, 1), (1, L.F64, 77777, 3), (2, L.F64, 1 << 18, 2),
    (0, L.I32, 1 << 20, 1), (1, L.I32, 4099, 5), (2, L.I32, 1 << 17, 1),
    (0, L.U32, 1 << 20, 1), (2, L.U32, 1 << 18, 1), (1, L.U32, 9, 1),
    # many slots: at most 8192 partials, so at most 2 blocks per slot at 4096 slots, 1 at 8192
    (0, L.F32, 1000, 4096), (2, L.I32, 64, 8192),
    # empty arrays: sum and dot are 0, mean is 0/0
    (0, L.F32, 0, 1), (1, L.F64, 0, 2), (2, L.U32, 0, 1),
]


@pytest.mark.parametrize("op,prec,n,slots", CASES)
def test_noalloc_reduce_matches_oracle_and_regular_entry_point(chai_dev, op, prec, n, slots):
    import torch
    lib = L.lib()
    rng = np.random.default_rng(11 + 7 * op + prec + n % 97 + slots)
    a_h = make(prec, max(1, n * slots), rng)
    b_h = make(prec, max(1, n * slots), rng)
    want, mag = oracle_reduce(op, prec, a_h, b_h, n, slots)
    a = torch.from_numpy(a_h.view(np.int32) if prec == L.U32 else a_h).cuda()
    b = torch.from_numpy(b_h.view(np.int32) if prec == L.U32 else b_h).cuda()
    # chai_cuda_reduce stages results in 4096 pinned doubles: compare with it up to that many slots
    reg = regular(chai_dev, op, prec, a, b, n, slots) if n and slots <= 4096 else None
    out = torch.empty(slots, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for call in range(2):
        out.fill_(12345.0)
        st = lib.chai_cuda_reduce_noalloc(op, prec, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), n, slots,
                                          C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == 0, (op, prec, n, slots, call, st)
        got = out.cpu().numpy()
        assert agree(op, prec, got, want, mag), (op, prec, n, slots, call, got[:4], want[:4])
        if reg is not None:
            assert agree(op, prec, got, reg, mag), (op, prec, n, slots, call, got[:4], reg[:4])


def test_noalloc_reduce_rejects_too_many_slots(chai_dev):
    import torch
    a = torch.zeros(8193, dtype=torch.float32, device="cuda")
    out = torch.zeros(8193, dtype=torch.float64, device="cuda")
    st = L.lib().chai_cuda_reduce_noalloc(0, 4, C.c_void_p(a.data_ptr()), None, 1, 8193, C.c_void_p(out.data_ptr()),
                                          None)
    assert st == -2
    st = L.lib().chai_cuda_reduce_noalloc(7, 4, C.c_void_p(a.data_ptr()), None, 1, 1, C.c_void_p(out.data_ptr()),
                                          None)
    assert st == -1
