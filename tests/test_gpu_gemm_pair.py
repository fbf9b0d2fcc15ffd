"""The CTA-pair tensor-core GEMM (tcgen05.mma.cta_group::2, 256-row tiles on
two SMs; the default for M > 128) against the one-CTA kernel (GemmPair=0)
and the FP64 oracle.

- Plain bf16 and tf32: every output element is the same sequence of 16-deep
  (8-deep) tensor-core accumulations in both kernels, so C is bit-identical.
- Split precisions (bf16x3, bf16x6): the pair kernel restarts the a0*b0
  accumulator every 4 K chunks and adds the segment sums in FP32 registers,
  so C differs from the one-CTA kernel in the last bits; both stay within
  the bounds of test_gpu_gemm.py, and the pair kernel's error is no larger
  than 1.25x the one-CTA kernel's (ragged shapes, alpha/beta, batches, M just
  above 128 and 256, K from one chunk to many segments).
Error metric: max |C - C64| / (|A||B|)_ij against oracle.gemm_f64."""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
BOUND = {L.GEMM_BF16: 2.0 ** -7, L.GEMM_TF32: 2.0 ** -9, L.GEMM_BF16X3: 2.0 ** -14, L.GEMM_BF16X6: 2.0 ** -20}


@pytest.fixture(scope="module")
def one_cta(chai_dev):
    import chai_b200.api as ch
    dev = ch.Device(config="GemmPair=0")
    yield dev
    dev.close()


def gemm(dev, A, B, prec, alpha=1.0, beta=0.0, C0=None):
    import torch
    batch = A.shape[0] if A.ndim == 3 else 1
    A3, B3 = A.reshape(batch, *A.shape[-2:]), B.reshape(batch, *B.shape[-2:])
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


def norm_err(Cg, A, B, alpha=1.0, beta=0.0, C0=None):
    want = alpha * oracle.gemm_f64(A, B)
    bound = abs(alpha) * (np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64))
    if C0 is not None:
        want = want + beta * C0.astype(np.float64)
        bound = bound + abs(beta) * np.abs(C0).astype(np.float64)
    return float(np.max(np.abs(Cg.astype(np.float64) - want) / np.maximum(bound, 1e-300)))


SHAPES = [(129, 200, 64), (256, 256, 256), (257, 300, 1000), (600, 520, 96), (384, 1000, 2048), (1024, 768, 4160)]


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_TF32])
@pytest.mark.parametrize("shape", SHAPES)
def test_pair_plain_bit_identical_to_one_cta(chai_dev, one_cta, prec, shape):
    M, N, K = shape
    rng = np.random.default_rng(M + 7 * N + K)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    got = gemm(chai_dev, A, B, prec)
    ref = gemm(one_cta, A, B, prec)
    assert np.array_equal(got, ref)
    assert norm_err(got, A, B) <= BOUND[prec]


@pytest.mark.parametrize("prec", [L.GEMM_BF16X3, L.GEMM_BF16X6])
@pytest.mark.parametrize("shape", SHAPES)
def test_pair_split_accuracy(chai_dev, one_cta, prec, shape):
    M, N, K = shape
    rng = np.random.default_rng(M + 5 * N + K)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    e_pair = norm_err(gemm(chai_dev, A, B, prec), A, B)
    e_one = norm_err(gemm(one_cta, A, B, prec), A, B)
    assert e_pair <= BOUND[prec] and e_pair <= 1.25 * e_one + 2.0 ** -24, (e_pair, e_one)


@pytest.mark.parametrize("prec", [L.GEMM_BF16, L.GEMM_BF16X3])
def test_pair_alpha_beta_batch(chai_dev, one_cta, prec):
    rng = np.random.default_rng(17)
    batch, M, N, K = 3, 300, 260, 520
    A = rng.uniform(-1, 1, (batch, M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (batch, K, N)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (batch, M, N)).astype(np.float32)
    got = gemm(chai_dev, A, B, prec, alpha=0.5, beta=-2.0, C0=C0)
    for i in range(batch):
        assert norm_err(got[i], A[i], B[i], 0.5, -2.0, C0[i]) <= BOUND[prec], i
    if prec == L.GEMM_BF16:
        assert np.array_equal(got, gemm(one_cta, A, B, prec, alpha=0.5, beta=-2.0, C0=C0))


def test_pair_sentinel(chai_dev):
    """A = B = 1: every entry equals K exactly (split: the a1 planes are 0)."""
    M, N, K = 512, 768, 1280
    for prec in (L.GEMM_BF16, L.GEMM_BF16X3, L.GEMM_BF16X6, L.GEMM_TF32):
        Cg = gemm(chai_dev, np.ones((M, K), np.float32), np.ones((K, N), np.float32), prec)
        assert np.all(Cg == K), prec
