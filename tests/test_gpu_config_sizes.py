"""Parity at the benchmark configurations' own sizes, through the C ABI.

- GEMM (the precision sweep): square bf16x3 and bf16x6 GEMMs at 4096^3
  (every entry), 8192^3 and 16384^3 (4096 sampled entries), on uniform[-1, 1)
  and N(0, 1) operands from the library's Philox fill (seeds 1, 2 and 3, 4;
  the rare +-inf normals of a u = 0 draw zeroed).  Error = max |C - C64| /
  (|A||B|)_ij, the componentwise-normalised relative error, against the FP64
  oracle (oracle.gemm_entries_f64, the interpreter's matmul in double,
  interp/InterpMatmulBase.hpp:50-61).  At 4096^3 the FP64 product of every
  entry comes from a cuBLAS DGEMM on the device, itself pinned to the oracle
  on 2048 sampled entries within 1e-12 relative.  Bound: 1e-6 -- the FP32-level
  accuracy the split precisions claim -- for both.
- Monte Carlo trace: 2^26 Philox4x32-10 Box-Muller pairs with seed 42
  (W = 8192, H = 16384); all 2^27 uniforms bit-exact against the oracle, all
  normals within 1e-5 * max(1, r) (f32 log / sincos on the device against
  double on the host); the payoff of the configured trace (+inf on both
  sides: a handful of u = 0 draws give infinite normals, as in the reference)
  and of the same trace with Z clamped to [-20, 20] (finite) within 1e-5
  relative.
- Kirsch 8-direction compass filter on an 8192 x 8192 uniform[0, 1) image
  (Philox seed 5): bit-exact against oracle.kirsch (interp/InterpGather.hpp:
  31-44 periodic wrap).
- GEMV 8192 x 8192, f32 and f64, against the FP64 oracle (oracle.gemv_f64):
  componentwise-normalised error <= 2^-20 (f32) and 2^-45 (f64).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32
FP32_LEVEL = 1e-6


@pytest.fixture()
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


def operands(dev, n, dist):
    """f32 n x n operands from the library's Philox fill, chai layout."""
    import torch
    out = []
    for seed in ((1, 2) if dist == "uniform" else (3, 4)):
        t = torch.empty((n, n), device="cuda", dtype=torch.float32)
        if dist == "uniform":
            rd = L.chai_rng_desc(L.PHILOX, L.F32, 0, 4, seed, n, n, 1, 1, -1.0, 1.0)
        else:
            rd = L.chai_rng_desc(L.PHILOX, L.F32, 1, 4, seed, n, n, 1, 0, 0.0, 1.0)
        L.check(L.lib().chai_cuda_rng_fill(dev.ctx, C.byref(rd), C.c_void_p(t.data_ptr())), dev.ctx)
        if dist == "normal":
            t.nan_to_num_(nan=0.0, posinf=0.0, neginf=0.0)
        out.append(t)
    return out


def gemm(dev, A, B, prec):
    import torch
    n = A.shape[0]
    Cm = torch.full((n, n), float("nan"), device="cuda", dtype=torch.float32)
    d = L.chai_gemm_desc(prec, 0, 0, 0, n, n, n, A.data_ptr(), n, B.data_ptr(), n, Cm.data_ptr(), n, 1.0, 0.0, 1,
                         0, 0, 0)
    L.check(L.lib().chai_cuda_gemm(dev.ctx, C.byref(d)), dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
    return Cm


def sampled_error(A, B, Cm, samples=4096, seed=0):
    """Normalised error on sampled entries against the FP64 oracle."""
    n = A.shape[0]
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n, samples)
    cols = rng.integers(0, n, samples)
    Ah, Bh = A.cpu().numpy(), B.cpu().numpy()
    c64 = oracle.gemm_entries_f64(Ah, Bh, rows, cols)
    bound = oracle.gemm_entries_f64(np.abs(Ah), np.abs(Bh), rows, cols)
    got = Cm.cpu().numpy()[rows, cols].astype(np.float64)
    return float(np.max(np.abs(got - c64) / bound))


@pytest.mark.parametrize("dist", ["uniform", "normal"])
@pytest.mark.parametrize("prec", [L.GEMM_BF16X3, L.GEMM_BF16X6])
def test_gemm_4096_every_entry(chai_dev, prec, dist):
    import torch
    n = 4096
    A, B = operands(chai_dev, n, dist)
    Cm = gemm(chai_dev, A, B, prec)
    A64, B64 = A.double(), B.double()
    C64 = A64 @ B64
    bound = A64.abs() @ B64.abs()
    # pin the device FP64 product to the oracle on sampled entries
    rng = np.random.default_rng(5)
    rows, cols = rng.integers(0, n, 2048), rng.integers(0, n, 2048)
    want = oracle.gemm_entries_f64(A.cpu().numpy(), B.cpu().numpy(), rows, cols)
    dev64 = C64.cpu().numpy()[rows, cols]
    assert np.all(np.abs(dev64 - want) <= 1e-12 * bound.cpu().numpy()[rows, cols])
    err = float(((Cm.double() - C64).abs() / bound).max())
    assert torch.isfinite(Cm).all()
    assert err <= FP32_LEVEL, (prec, dist, err)


@pytest.mark.parametrize("n", [8192, 16384])
@pytest.mark.parametrize("dist", ["uniform", "normal"])
@pytest.mark.parametrize("prec", [L.GEMM_BF16X3, L.GEMM_BF16X6])
def test_gemm_large_sampled(chai_dev, prec, dist, n):
    import torch
    A, B = operands(chai_dev, n, dist)
    Cm = gemm(chai_dev, A, B, prec)
    assert bool(torch.isfinite(Cm).all())
    err = sampled_error(A, B, Cm)
    del A, B, Cm
    torch.cuda.empty_cache()
    assert err <= FP32_LEVEL, (prec, dist, n, err)


MC_W, MC_H = 8192, 16384          # 2^27 normals from 2^26 Box-Muller pairs


def test_mc_uniforms_and_normals_full_size(ch):
    g = ch.RNGf32(ch.RNG_PHILOX, 42)
    u = ch.Arrayf32(ch.rng_uniform_make(g, MC_W, MC_H)).read1()
    want_u = oracle.rng_fill(MC_W * MC_H, seed=42)
    assert np.array_equal(u, want_u)
    del u
    g = ch.RNGf32(ch.RNG_PHILOX, 42)
    z = ch.Arrayf32(ch.rng_normal_make(g, MC_W, MC_H)).read1()
    want_z = oracle.rng_fill(MC_W * MC_H, dist=1, seed=42)
    # equal values include the +-inf of u = 0 draws; the rest within the bound
    idx = np.nonzero(z != want_z)[0]
    u0 = want_u.reshape(-1, 2)[idx // 2, 0].astype(np.float64)
    r = np.sqrt(-2.0 * np.log(u0))
    dz = np.abs(z[idx].astype(np.float64) - want_z[idx].astype(np.float64))
    assert np.all(dz <= 1e-5 * np.maximum(1.0, r)), (idx[:8], dz.max())


def mc_trace(ch, clamp):
    g = ch.RNGf32(ch.RNG_PHILOX, 42)
    Z = ch.rng_normal_make(g, MC_W, MC_H)
    if clamp:
        Z = ch.min(ch.max(Z, f32(-20)), f32(20))
    S = f32(100) * ch.exp(f32(0.05 - 0.5 * 0.2 * 0.2) + f32(0.2) * Z)
    return float(ch.Arrayf32(ch.mean(ch.max(S - f32(100), f32(0)))).read_scalar())


def mc_oracle(z, clamp):
    z = z.astype(np.float32)
    if clamp:
        z = np.minimum(np.maximum(z, f32(-20)), f32(20))
    with np.errstate(over="ignore", invalid="ignore"):
        s = f32(100) * np.exp(f32(0.05 - 0.5 * 0.2 * 0.2) + f32(0.2) * z)
        return float(np.maximum(s - f32(100), f32(0)).astype(np.float64).mean())


def test_mc_payoff_full_size(ch):
    z = oracle.rng_fill(MC_W * MC_H, dist=1, seed=42)
    want = mc_oracle(z, False)
    got = mc_trace(ch, False)
    assert got == want or abs(got - want) <= 1e-5 * abs(want), (got, want)
    want_c = mc_oracle(z, True)
    got_c = mc_trace(ch, True)
    assert np.isfinite(want_c) and abs(got_c - want_c) <= 1e-5 * abs(want_c), (got_c, want_c)


def test_kirsch_8192_bit_exact(ch):
    from tests.test_gpu_trace import kirsch_expr
    W = H = 8192
    img = oracle.rng_fill(W * H, seed=5).reshape(H, W)
    A = ch.make2(img)
    got = ch.Arrayf32(kirsch_expr(ch, A, W, H)).read2()
    assert np.array_equal(got, oracle.kirsch(img))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gemv_8192(chai_dev, dtype):
    import torch
    n = 8192
    rng = np.random.default_rng(8192)
    A = rng.uniform(-1, 1, (n, n)).astype(dtype)
    x = rng.uniform(-1, 1, n).astype(dtype)
    a, xv = torch.from_numpy(A).cuda(), torch.from_numpy(x).cuda()
    y = torch.full((n,), float("nan"), dtype=a.dtype, device="cuda")
    prec = L.F32 if dtype == np.float32 else L.F64
    L.check(L.lib().chai_cuda_gemv(chai_dev.ctx, prec, 0, n, n, 1.0, a.data_ptr(), n, xv.data_ptr(), 0.0,
                                   y.data_ptr()), chai_dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(chai_dev.ctx), chai_dev.ctx)
    want = oracle.gemv_f64(A, x)
    bound = oracle.gemv_f64(np.abs(A), np.abs(x))
    err = np.max(np.abs(y.cpu().numpy().astype(np.float64) - want) / bound)
    assert err <= (2.0 ** -20 if dtype == np.float32 else 2.0 ** -45), err
