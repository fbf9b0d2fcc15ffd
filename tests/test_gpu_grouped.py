"""Grouped GEMM: many independent f32 problems of different shapes in one
persistent tcgen05 launch (chai_cuda_gemm_grouped), each checked against the
FP64 oracle with the componentwise-normalised error of test_gpu_gemm.py
(bf16x3: 2^-14, bf16: 2^-7, bf16x6: 2^-20)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
BOUND = {L.GEMM_BF16: 2.0 ** -7, L.GEMM_BF16X3: 2.0 ** -14, L.GEMM_BF16X6: 2.0 ** -20}


def problems(count, seed=11, lo=32, hi=512):
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.integers(lo // 8, hi // 8 + 1, 3) * 8) for _ in range(count)]


def run_grouped(dev, shapes, prec, seed=1):
    import torch
    rng = np.random.default_rng(seed)
    As = [rng.uniform(-1, 1, (m, k)).astype(np.float32) for m, n, k in shapes]
    Bs = [rng.uniform(-1, 1, (k, n)).astype(np.float32) for m, n, k in shapes]
    ta = [torch.from_numpy(a).cuda() for a in As]
    tb = [torch.from_numpy(b).cuda() for b in Bs]
    tc = [torch.full((m, n), float("nan"), device="cuda") for m, n, k in shapes]
    arr = (L.chai_gemm_problem * len(shapes))()
    for i, (m, n, k) in enumerate(shapes):
        arr[i] = L.chai_gemm_problem(m, n, k, 0, ta[i].data_ptr(), tb[i].data_ptr(), tc[i].data_ptr())
    L.check(L.lib().chai_cuda_gemm_grouped(dev.ctx, prec, arr, len(shapes)), dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
    return As, Bs, [c.cpu().numpy() for c in tc]


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_BF16X3, L.GEMM_BF16X6])
def test_grouped_gemm_vs_fp64(chai_dev, prec):
    shapes = problems(48) + [(8, 8, 8), (513 // 8 * 8, 8, 504), (40, 512, 32)]
    As, Bs, Cs = run_grouped(chai_dev, shapes, prec)
    worst = 0.0
    for a, b, c in zip(As, Bs, Cs):
        c64 = oracle.gemm_f64(a, b)
        bound = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64)
        worst = max(worst, float(np.max(np.abs(c - c64) / bound)))
    assert worst <= BOUND[prec], worst


def test_grouped_gemm_4096_problems_sample(chai_dev):
    """The full 4096-problem group (M, N, K multiples of 8 in [32, 512],
    seed 11); every 97th problem is checked against the FP64 oracle."""
    shapes = problems(4096)
    As, Bs, Cs = run_grouped(chai_dev, shapes, L.GEMM_BF16X3)
    for i in range(0, 4096, 97):
        c64 = oracle.gemm_f64(As[i], Bs[i])
        bound = np.abs(As[i]).astype(np.float64) @ np.abs(Bs[i]).astype(np.float64)
        assert np.max(np.abs(Cs[i] - c64) / bound) <= BOUND[L.GEMM_BF16X3], i


def fused_count(dev):
    """Grouped GEMMs of this context that split their operands in-kernel."""
    ms, n = C.c_double(), C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(dev.ctx, b"grouped_fused", C.byref(ms), C.byref(n), 0), dev.ctx)
    return n.value


@pytest.fixture(scope="module")
def prepass_dev(chai_dev):
    """A second context whose grouped GEMM writes the bf16 planes in a prepass."""
    import chai_b200.api as ch
    dev = ch.Device(config="GroupedSplit=prepass")
    yield dev
    dev.close()


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_BF16X3, L.GEMM_BF16X6])
def test_in_kernel_split_equals_prepass_planes(chai_dev, prepass_dev, prec):
    """The fused kernel splits f32 tiles in shared memory; the prepass path
    writes the planes to HBM first.  Both issue the same planes, products and
    accumulators per element, so C must be bit-identical (K tails of 8, 36,
    100 elements; M and N past a tile edge)."""
    shapes = problems(40, seed=5) + [(8, 8, 8), (136, 260, 100), (129, 132, 36), (300, 4, 2056), (68, 44, 20),
                                     (3, 128, 4)]
    before = fused_count(chai_dev)
    _, _, fused = run_grouped(chai_dev, shapes, prec, seed=3)
    assert fused_count(chai_dev) == before + 1          # the in-kernel split ran
    _, _, pre = run_grouped(prepass_dev, shapes, prec, seed=3)
    assert fused_count(prepass_dev) == 0
    for i, (a, b) in enumerate(zip(fused, pre)):
        assert np.array_equal(a, b), (i, shapes[i])


def test_unaligned_group_falls_back_to_prepass(chai_dev):
    """K = 42 rows of A cannot be read in 16-byte loads: the whole group takes
    the prepass path and stays within the bf16x3 bound."""
    shapes = [(64, 40, 42), (96, 64, 72)]
    before = fused_count(chai_dev)
    As, Bs, Cs = run_grouped(chai_dev, shapes, L.GEMM_BF16X3)
    assert fused_count(chai_dev) == before
    for a, b, c in zip(As, Bs, Cs):
        bound = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64)
        assert np.max(np.abs(c - oracle.gemm_f64(a, b)) / bound) <= BOUND[L.GEMM_BF16X3]


def test_unaligned_c_uses_scalar_stores(chai_dev, prepass_dev):
    """C one float past a 16-byte boundary (A and B aligned, K and N multiples
    of 4): the in-kernel split still runs, its epilogue stores C element by
    element instead of through the shared-memory stage, and C equals the
    prepass path's bit for bit; the float before C is left alone."""
    import torch
    shapes = [(136, 260, 100), (40, 128, 36), (300, 44, 64)]
    rng = np.random.default_rng(8)
    outs = []
    for dev in (chai_dev, prepass_dev):
        ta = [torch.from_numpy(rng.uniform(-1, 1, (m, k)).astype(np.float32)).cuda() for m, n, k in shapes]
        tb = [torch.from_numpy(rng.uniform(-1, 1, (k, n)).astype(np.float32)).cuda() for m, n, k in shapes]
        rng = np.random.default_rng(8)                      # same operands for both paths
        tc = [torch.full((m * n + 1,), -7.0, device="cuda") for m, n, k in shapes]
        arr = (L.chai_gemm_problem * len(shapes))()
        for i, (m, n, k) in enumerate(shapes):
            arr[i] = L.chai_gemm_problem(m, n, k, 0, ta[i].data_ptr(), tb[i].data_ptr(), tc[i].data_ptr() + 4)
        before = fused_count(dev)
        L.check(L.lib().chai_cuda_gemm_grouped(dev.ctx, L.GEMM_BF16X3, arr, len(shapes)), dev.ctx)
        L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
        assert fused_count(dev) == before + (1 if dev is chai_dev else 0)
        outs.append([c.cpu().numpy() for c in tc])
    for (m, n, k), a, b in zip(shapes, outs[0], outs[1]):
        assert a[0] == -7.0 and np.array_equal(a, b), (m, n, k)


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_BF16X3])
def test_tma_b_equals_register_b(chai_dev, prec):
    """B through TMA (raw f32 boxes of 64 k x 128 n, zero-filled past N and
    K, split from shared memory) against B loaded into the converters'
    registers (the default): the same planes, so C is bit-identical,
    including a K > 2048 problem (two accumulators) and N of 4."""
    import chai_b200.api as ch
    shapes = problems(40, seed=9) + [(136, 260, 100), (129, 132, 36), (300, 4, 2056), (68, 44, 20), (3, 128, 4)]
    _, _, reg = run_grouped(chai_dev, shapes, prec, seed=4)
    dev = ch.Device(config="GroupedTmaB=1")
    try:
        before = fused_count(dev)
        _, _, bt = run_grouped(dev, shapes, prec, seed=4)
        assert fused_count(dev) == before + 1
    finally:
        dev.close()
    for i, (a, b) in enumerate(zip(bt, reg)):
        assert np.array_equal(a, b), (i, shapes[i])


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_BF16X3])
def test_pair_tiles_equal_one_cta_kernel(chai_dev, prec):
    """256 x 256 output tiles on CTA pairs (tcgen05.mma.cta_group::2, each
    CTA converting half of A's rows and half of B's columns) against the
    one-CTA kernel's 128 x 128 tiles (GroupedPair=0): the same per-element
    product sequence, so C is bit-identical -- M and N below, at and past
    the 256 edge, N of 4, K tails."""
    import chai_b200.api as ch
    shapes = problems(60, seed=17) + [(256, 256, 64), (257, 260, 72), (128, 512, 100), (512, 128, 36), (3, 4, 4),
                                      (300, 4, 200), (8, 520, 8), (264, 8, 512)]
    _, _, pair = run_grouped(chai_dev, shapes, prec, seed=7)
    dev = ch.Device(config="GroupedPair=0")
    try:
        _, _, one = run_grouped(dev, shapes, prec, seed=7)
    finally:
        dev.close()
    for i, (a, b) in enumerate(zip(pair, one)):
        assert np.array_equal(a, b), (i, shapes[i])
