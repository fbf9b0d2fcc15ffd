"""GEMM precision sweep parity: every arithmetic of chai_cuda_gemm against the
FP64 oracle (oracle/ops.c, pinned to the reference interpreter's matmul).

Error metric (stated per precision): max |C - C64| / (|A| |B|)_ij, the
componentwise-bound-normalised error, and the reference autotuner's two
self-checks (autotune/EvergreenMatmulMM.cpp:905-1000): the sentinel (A = B = 1
gives C = K) and the "paranoid" L1 check against a CPU double reference.

Bounds: bf16 2^-7, tf32 2^-9 (operands keep 10 mantissa bits), bf16x3 2^-14
(dropped a1*b1 and residual terms ~2^-16), bf16x6 within 4x the FP32 SIMT
GEMM's own error plus 2^-22 (FP32 accumulation dominates), fp32 SIMT 2^-18,
fp8 e4m3 with per-tile scales 2^-4 (3 mantissa bits: each operand is off by
at most 2^-4 of its tile's scale-relative magnitude)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu

BOUND = {L.GEMM_BF16: 2.0 ** -7, L.GEMM_TF32: 2.0 ** -9, L.GEMM_BF16X3: 2.0 ** -14, L.GEMM_FP32: 2.0 ** -18,
         L.GEMM_FP8: 2.0 ** -4}


def run_gemm(dev, A, B, prec, alpha=1.0, beta=0.0, C0=None):
    import torch
    batch = A.shape[0] if A.ndim == 3 else 1
    A3 = A.reshape(batch, *A.shape[-2:])
    B3 = B.reshape(batch, *B.shape[-2:])
    M, K = A3.shape[1:]
    N = B3.shape[2]
    a = torch.from_numpy(np.ascontiguousarray(A3)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(B3)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(C0.reshape(batch, M, N))).cuda() if C0 is not None else \
        torch.full((batch, M, N), float("nan"), device="cuda")
    d = L.chai_gemm_desc(prec, 0, 0, 0, M, N, K, a.data_ptr(), K, b.data_ptr(), N, c.data_ptr(), N, alpha, beta,
                         batch, M * K, K * N, M * N)
    L.check(L.lib().chai_cuda_gemm(dev.ctx, C.byref(d)), dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
    return c.cpu().numpy().reshape(A.shape[:-2] + (M, N))


def norm_err(Cg, A, B):
    C64 = oracle.gemm_f64(A, B)
    bound = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    return float(np.max(np.abs(Cg.astype(np.float64) - C64) / np.maximum(bound, 1e-300)))


SHAPES = [(128, 256, 64), (200, 300, 100), (512, 512, 512), (256, 384, 2048), (1, 17, 9)]


@pytest.mark.parametrize("prec", [L.GEMM_FP32, L.GEMM_BF16, L.GEMM_TF32, L.GEMM_BF16X3, L.GEMM_BF16X6, L.GEMM_FP8])
@pytest.mark.parametrize("shape", SHAPES)
def test_gemm_precision_vs_fp64(chai_dev, prec, shape):
    M, N, K = shape
    A = oracle.rng_fill(M * K, seed=1, limits=(-1.0, 1.0)).reshape(M, K)
    B = oracle.rng_fill(K * N, seed=2, limits=(-1.0, 1.0)).reshape(K, N)
    Cg = run_gemm(chai_dev, A, B, prec)
    e = norm_err(Cg, A, B)
    if prec == L.GEMM_BF16X6:
        e32 = norm_err(run_gemm(chai_dev, A, B, L.GEMM_FP32), A, B)
        assert e <= 4 * e32 + 2.0 ** -22, (e, e32)
    else:
        assert e <= BOUND[prec], e


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_TF32, L.GEMM_BF16X3, L.GEMM_BF16X6])
def test_gemm_sentinel(chai_dev, prec):
    """A = B = 1: every entry of C equals K exactly (sentinel check)."""
    M, N, K = 256, 512, 768
    Cg = run_gemm(chai_dev, np.ones((M, K), np.float32), np.ones((K, N), np.float32), prec)
    assert np.all(Cg == K)


def test_fp8_sentinel(chai_dev):
    """A = B = 1: e4m3(448) * e4m3(448) * (1/448)^2 summed K times -> K to one
    rounding of the dequantisation scale."""
    M, N, K = 256, 512, 768
    Cg = run_gemm(chai_dev, np.ones((M, K), np.float32), np.ones((K, N), np.float32), L.GEMM_FP8)
    assert np.all(np.abs(Cg - K) <= 2.0 ** -20 * K)


def test_fp8_per_tile_scales(chai_dev):
    """Row tiles of A and column blocks of B with magnitudes 10^-3 .. 10^3: a
    scale per 128-row tile of A and per 128-column block of B keeps the error
    relative to each tile's own magnitude (a single scale would flush the
    small tiles to zero)."""
    rng = np.random.default_rng(21)
    M, N, K = 384, 520, 200
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    A *= np.repeat(10.0 ** np.array([-3.0, 0.0, 3.0]), 128)[:, None].astype(np.float32)
    B *= np.repeat(10.0 ** np.array([2.0, -2.0, 0.0, 1.0, -3.0]), 128)[None, :N].astype(np.float32)
    Cg = run_gemm(chai_dev, A, B, L.GEMM_FP8)
    assert norm_err(Cg, A, B) <= 2.0 ** -4


@pytest.mark.parametrize("prec", [L.GEMM_BF16X3, L.GEMM_TF32, L.GEMM_FP8])
def test_gemm_alpha_beta_batch(chai_dev, prec):
    """C = alpha A B + beta C over a strided batch (matmulG over vector slots)."""
    rng = np.random.default_rng(9)
    batch, M, N, K = 3, 130, 260, 96
    A = rng.uniform(-1, 1, (batch, M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (batch, K, N)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (batch, M, N)).astype(np.float32)
    Cg = run_gemm(chai_dev, A, B, prec, alpha=0.5, beta=-2.0, C0=C0)
    for i in range(batch):
        want = 0.5 * oracle.gemm_f64(A[i], B[i]) - 2.0 * C0[i].astype(np.float64)
        bound = 0.5 * (np.abs(A[i]).astype(np.float64) @ np.abs(B[i])) + 2.0 * np.abs(C0[i])
        assert np.max(np.abs(Cg[i] - want) / bound) <= BOUND[prec]


@pytest.mark.parametrize("prec", [L.GEMM_FP32, L.GEMM_BF16X6])
def test_gemm_paranoid_l1(chai_dev, prec):
    """The reference autotuner's paranoid check (EvergreenMatmulMM.cpp:
    945-1040): inputs uniform on [0, 1), L1 distance to the CPU double result
    below 1 (devspec.cfg Paranoid=1 on GPUs) and the mean of C within 10% of
    K/4.  An FP32-level check, so it applies to fp32 and bf16x6."""
    rng = np.random.default_rng(3)
    n = 128
    A = rng.uniform(0, 1, (n, n)).astype(np.float32)
    B = rng.uniform(0, 1, (n, n)).astype(np.float32)
    Cg = run_gemm(chai_dev, A, B, prec)
    assert np.abs(Cg - oracle.gemm_f64(A, B)).sum() < 1.0
    assert abs(Cg.mean() - 0.25 * n) / (0.25 * n) < 0.1


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(1, 4), (37, 4096), (300, 8192), (1000, 4100), (5, 20000)])
def test_gemv_bulk_copy_path(chai_dev, dtype, shape):
    """The cp.async.bulk GEMV (16-byte aligned A, x, pitch and row length):
    rows shorter than one 16 KB chunk, exactly one, several, a ragged last
    chunk; alpha and beta applied once.  Against the FP64 product,
    componentwise-normalised: 2^-20 (f32), 2^-45 (f64)."""
    import torch
    m, n = shape
    rng = np.random.default_rng(m + n)
    A = rng.uniform(-1, 1, (m, n)).astype(dtype)
    x = rng.uniform(-1, 1, n).astype(dtype)
    y0 = rng.uniform(-1, 1, m).astype(dtype)
    a, xv, y = torch.from_numpy(A).cuda(), torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
    prec = L.F32 if dtype == np.float32 else L.F64
    L.check(L.lib().chai_cuda_gemv(chai_dev.ctx, prec, 0, m, n, 0.5, a.data_ptr(), n, xv.data_ptr(), -2.0,
                                   y.data_ptr()), chai_dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(chai_dev.ctx), chai_dev.ctx)
    want = 0.5 * (A.astype(np.float64) @ x.astype(np.float64)) - 2.0 * y0.astype(np.float64)
    bound = 0.5 * (np.abs(A).astype(np.float64) @ np.abs(x).astype(np.float64)) + 2.0 * np.abs(y0)
    err = np.max(np.abs(y.cpu().numpy().astype(np.float64) - want) / bound)
    assert err <= (2.0 ** -20 if dtype == np.float32 else 2.0 ** -45), err


@pytest.mark.parametrize("shape", [(512, 512, 512), (256, 264, 40), (1024, 512, 96)])
def test_fp32_gemm_tile_choice_is_bit_identical(chai_dev, shape):
    """The FP32 CUDA-core GEMM picks 128x128, 64x64 or 32x64 tiles by how many
    tiles cover the SMs; each output's FMA chain runs in the same k order in
    every variant, so a small product (few tiles, small-tile kernel) equals
    the same product as entry 0 of a 10-problem batch (enough tiles for the
    128x128 kernel) bit for bit."""
    M, N, K = shape
    rng = np.random.default_rng(M + N + K)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    one = run_gemm(chai_dev, A, B, L.GEMM_FP32)
    many = run_gemm(chai_dev, np.repeat(A[None], 10, 0), np.repeat(B[None], 10, 0), L.GEMM_FP32)
    assert np.array_equal(one, many[0]) and np.array_equal(many[0], many[9])
    assert norm_err(one, A, B) <= BOUND[L.GEMM_FP32]
