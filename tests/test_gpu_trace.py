"""GPU parity of the trace path (RNG, fused element kernels, reductions,
gathers) against the oracle.  Tolerances are written next to each check.

Bit-exact: integer arrays, raw Random123 lanes, f32/f64 uniforms, gather
indices (Kirsch output is compared exactly because every term is an exact
f32 operation on the same inputs in the same order).
Floating point: normals within 1e-5 * max(1, |r|) absolute (f32 log / sincos of
the device vs double on the host), transcendental element ops within 4 ulp-ish
relative bounds stated per op, reductions within 1e-12 relative of the FP64
oracle (FP64 accumulation on both sides, different order)."""
import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.fixture()
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


# ----------------------------------------------------------------- RNG

@pytest.mark.parametrize("variant", [oracle.PHILOX, oracle.THREEFRY])
@pytest.mark.parametrize("prec", [oracle.U32, oracle.I32, oracle.F32, oracle.F64])
def test_rng_uniform_bit_exact(ch, variant, prec):
    G = {oracle.U32: ch.RNGu32, oracle.I32: ch.RNGi32, oracle.F32: ch.RNGf32, oracle.F64: ch.RNGf64}[prec]
    g = G(variant, 12345)
    W, H = 96, 37
    a = ch.Array.__new__(ch._ARR[prec])
    a = ch._ARR[prec](ch.rng_uniform_make(g, W, H))
    got = a.read1()
    want = oracle.rng_fill(W * H, variant=variant, prec=prec, seed=12345,
                           limits=(0.0, 1.0) if prec in (oracle.F32, oracle.F64) else None)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
    assert g.seed == (12345 + W * H) & ((1 << (64 if prec == oracle.F64 else 32)) - 1)


@pytest.mark.parametrize("variant", [oracle.PHILOX, oracle.THREEFRY])
def test_rng_uniform_limits_f32(ch, variant):
    g = ch.RNGf32(variant, 7)
    a = ch.Arrayf32(ch.rng_uniform_make(g, 256, 64, 1, -1.0, 1.0))
    got = a.read1()
    want = oracle.rng_fill(256 * 64, variant=variant, prec=oracle.F32, seed=7, limits=(-1.0, 1.0))
    assert np.array_equal(got, want)
    # the reference's interval is closed: values stay in [-1, 1]
    assert got.min() >= -1.0 and got.max() <= 1.0


@pytest.mark.parametrize("variant", [oracle.PHILOX, oracle.THREEFRY])
@pytest.mark.parametrize("prec", [oracle.F32, oracle.F64])
def test_rng_normal(ch, variant, prec):
    G = ch.RNGf32 if prec == oracle.F32 else ch.RNGf64
    g = G(variant, 99)
    W, H = 128, 40
    got = ch._ARR[prec](ch.rng_normal_make(g, W, H)).read1().astype(np.float64)
    want = oracle.rng_fill(W * H, variant=variant, prec=prec, dist=1, seed=99).astype(np.float64)
    u = oracle.rng_fill(W * H, variant=variant, prec=prec, seed=99).astype(np.float64)
    r = np.sqrt(-2.0 * np.log(np.repeat(u.reshape(-1, 2)[:, 0], 2)))
    tol = (1e-5 if prec == oracle.F32 else 1e-12) * np.maximum(1.0, r)
    assert np.all(np.abs(got - want) <= tol)


def test_rng_ragged_width(ch):
    """W not a multiple of the vector length: per-element generator calls on
    padded rows (vector index = y * ceil(W/4) + x/4)."""
    g = ch.RNGu32(ch.RNG_PHILOX, 3)
    W, H = 13, 5
    got = ch.Arrayu32(ch.rng_uniform_make(g, W, H)).read1().reshape(H, W)
    padded = oracle.rng_fill(16 * H, prec=oracle.U32, seed=3).reshape(H, 16)
    assert np.array_equal(got, padded[:, :W])


def test_rng_fill_direct_entry_point(ch, chai_dev):
    import ctypes as C
    import torch
    out = torch.empty(1 << 20, dtype=torch.float32, device="cuda")
    d = L.chai_rng_desc(oracle.PHILOX, oracle.F32, 0, 4, 42, 1024, 1024, 1, 1, -1.0, 1.0)
    L.check(L.lib().chai_cuda_rng_fill(chai_dev.ctx, C.byref(d), C.c_void_p(out.data_ptr())), chai_dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(chai_dev.ctx), chai_dev.ctx)
    want = oracle.rng_fill(1 << 20, seed=42, limits=(-1.0, 1.0))
    assert np.array_equal(out.cpu().numpy(), want)


# ----------------------------------------------------------- fused traces

def test_monte_carlo_trace_fused(ch):
    """S = 100 exp(0.03 + 0.2 Z), payoff = mean(max(S - 100, 0)) in one
    kernel; compared with the same arithmetic on the oracle's normals."""
    W, H = 1024, 512
    g = ch.RNGf32(ch.RNG_PHILOX, 42)
    p = ch.Arrayf32(ch.mean(ch.max(f32(100) * ch.exp(f32(0.03) + f32(0.2) * ch.rng_normal_make(g, W, H))
                                   - f32(100), f32(0))))
    got = float(p.read_scalar())
    z = oracle.rng_fill(W * H, dist=1, seed=42).astype(np.float32)
    s = f32(100) * np.exp(f32(0.03) + f32(0.2) * z)
    want = np.maximum(s - f32(100), f32(0)).astype(np.float64).mean()
    assert abs(got - want) <= 1e-5 * abs(want)


def test_monte_carlo_named_intermediates(ch):
    """Named arrays that stay alive are materialised (live variables) and the
    result is unchanged."""
    W, H = 256, 64
    g = ch.RNGf32(ch.RNG_PHILOX, 5)
    z = ch.Arrayf32(ch.rng_normal_make(g, W, H))
    s = ch.Arrayf32(f32(100) * ch.exp(f32(0.03) + f32(0.2) * z))
    p = ch.Arrayf32(ch.mean(ch.max(s - f32(100), f32(0))))
    got = float(p.read_scalar())
    zz = z.read1()
    want_z = oracle.rng_fill(W * H, dist=1, seed=5)
    assert np.allclose(zz, want_z, atol=1e-4)
    ss = s.read1()
    want = np.maximum(ss.astype(np.float64) - 100, 0).mean()
    assert abs(got - want) <= 1e-6 * abs(want) + 1e-7


def test_f64_promotion_of_double_literals(ch):
    """A C++ double literal promotes the expression to f64 (interp/InterpFun2.cpp:21);
    the assignment rounds back to f32."""
    x = np.linspace(-3, 3, 4096, dtype=np.float32)
    a = ch.make1(x)
    b = ch.Arrayf32(0.1 * a + 0.7)
    got = b.read1()
    want = (0.1 * x.astype(np.float64) + 0.7).astype(np.float32)
    assert np.array_equal(got, want)


ELEM1 = ["exp", "log", "sqrt", "sin", "cos", "tanh", "fabs", "floor", "ceil", "rsqrt", "log2", "exp2", "atan",
         "cbrt", "erf", "asinpi", "degrees", "sign"]


@pytest.mark.parametrize("name", ELEM1)
def test_unary_ops_f32(ch, name):
    x = np.linspace(0.05, 0.95, 1000, dtype=np.float32)
    got = ch.Arrayf32(getattr(ch, name)(ch.make1(x))).read1().astype(np.float64)
    xd = x.astype(np.float64)
    ref = {"exp": np.exp, "log": np.log, "sqrt": np.sqrt, "sin": np.sin, "cos": np.cos, "tanh": np.tanh,
           "fabs": np.abs, "floor": np.floor, "ceil": np.ceil, "rsqrt": lambda v: 1 / np.sqrt(v), "log2": np.log2,
           "exp2": np.exp2, "atan": np.arctan, "cbrt": np.cbrt, "erf": None, "asinpi": lambda v: np.arcsin(v) / np.pi,
           "degrees": np.degrees, "sign": np.sign}[name]
    if ref is None:
        import math
        want = np.array([math.erf(v) for v in xd])
    else:
        want = ref(xd)
    # CUDA's f32 functions: <= 4 ulp in this domain
    assert np.all(np.abs(got - want) <= 4 * np.spacing(np.abs(want).astype(np.float32)).astype(np.float64) + 1e-30)


def test_integer_ops_bit_exact(ch):
    rng = np.random.default_rng(0)
    a = rng.integers(-2**31, 2**31, 4096, dtype=np.int64).astype(np.int32)
    b = rng.integers(-2**31, 2**31, 4096, dtype=np.int64).astype(np.int32)
    A, B = ch.make1(a), ch.make1(b)
    got = {
        "add": ch.Arrayi32(A + B).read1(),
        "xor": ch.Arrayi32(A ^ B).read1(),
        "mul_hi": ch.Arrayi32(ch.mul_hi(A, B)).read1(),
        "add_sat": ch.Arrayi32(ch.add_sat(A, B)).read1(),
        "max": ch.Arrayi32(ch.max(A, B)).read1(),
        "lt": ch.Arrayi32(A < B).read1(),
        "rotate": ch.Arrayi32(ch.rotate(A, B & 31)).read1(),
    }
    a64, b64 = a.astype(np.int64), b.astype(np.int64)
    assert np.array_equal(got["add"], (a64 + b64).astype(np.int32))
    assert np.array_equal(got["xor"], a ^ b)
    assert np.array_equal(got["mul_hi"], ((a64 * b64) >> 32).astype(np.int32))
    assert np.array_equal(got["add_sat"], np.clip(a64 + b64, -2**31, 2**31 - 1).astype(np.int32))
    assert np.array_equal(got["max"], np.maximum(a, b))
    assert np.array_equal(got["lt"], (a < b).astype(np.int32))
    au = a.view(np.uint32).astype(np.uint64)
    r = (b & 31).astype(np.uint64)
    rot = (((au << r) | (au >> ((32 - r) % 32))) & 0xFFFFFFFF).astype(np.uint32)
    rot = np.where(r == 0, au.astype(np.uint32), rot)
    assert np.array_equal(got["rotate"].view(np.uint32), rot)


def test_cond_and_predicates(ch):
    x = np.linspace(-2, 2, 4000, dtype=np.float32)
    X = ch.make1(x)
    got = ch.Arrayf32(ch.cond(X > f32(0), X * f32(2), -X)).read1()
    assert np.array_equal(got, np.where(x > 0, x * f32(2), -x))


def test_index_zeros_ones(ch):
    W, H = 37, 11
    xi = ch.Arrayf32(ch.index_f32(0, W, H) + f32(10) * ch.index_f32(1, W, H) + ch.ones_f32(W, H)).read2()
    yy, xx = np.mgrid[0:H, 0:W]
    assert np.array_equal(xi, (xx + 10 * yy + 1).astype(np.float32))
    z = ch.Arrayf64(ch.zeros_f64(8, 4)).read1()
    assert not z.any()


def test_reductions_sum_mean_dot(ch):
    rng = np.random.default_rng(1)
    for n in (1, 3, 1000, 1 << 20, (1 << 20) + 7):
        a = rng.standard_normal(n).astype(np.float32)
        b = rng.standard_normal(n).astype(np.float32)
        A, B = ch.make1(a), ch.make1(b)
        s = float(ch.Arrayf64(ch.sum(ch.convert_f64(A))).read_scalar())
        ref = oracle.sum_f32(a)
        assert abs(s - ref) <= 1e-12 * max(1.0, np.abs(a).astype(np.float64).sum())
        m = float(ch.Arrayf32(ch.mean(A)).read_scalar())
        assert abs(m - np.float32(ref / n)) <= 2 * np.spacing(np.float32(abs(ref / n)))
        d = float(ch.Arrayf32(ch.dot_product(A, B)).read_scalar())
        refd = oracle.dot_f32(a, b)
        assert abs(d - np.float32(refd)) <= 2 * np.spacing(np.float32(abs(refd))) + 1e-30


def test_dot_product_terms_in_operand_type(ch):
    """dot_product forms each product in the operands' common C type before
    the FP64 sum (interp/InterpDotprod.cpp:40-138): f32 * f32 rounds to f32,
    i32 * i32 and u32 * u32 wrap in 32 bits."""
    e = np.float32(1 + 2.0 ** -12)
    # exact products: (1 + 2^-11 + 2^-24) - 1; the f32 product rounds the
    # 2^-24 away (ties to even), so the reference's result is 2^-11
    a = np.array([e, 1], dtype=np.float32)
    b = np.array([e, -1], dtype=np.float32)
    d = float(ch.Arrayf32(ch.dot_product(ch.make1(a), ch.make1(b))).read_scalar())
    assert d == oracle.dot_f32(a, b) == 2.0 ** -11
    # 70000^2 = 4.9e9 wraps to 605032704 in 32 bits
    for dt, arr in ((np.int32, ch.Arrayi32), (np.uint32, ch.Arrayu32)):
        x = np.array([70000, 3], dtype=dt)
        y = np.array([70000, 5], dtype=dt)
        want = int((np.int64(70000) * 70000) % (1 << 32)) + 15
        got = int(arr(ch.dot_product(ch.make1(x), ch.make1(y))).read_scalar())
        assert got == want == 605032719, (dt, got)


def test_reduce_accum_f32_stays_close(ch):
    """ReduceAccum=f32 (per-thread f32 partials) on a 2^22-element Monte Carlo
    mean: within 1e-6 relative of the FP64 default."""
    f32 = np.float32

    def payoff():
        g = ch.RNGf32(ch.RNG_PHILOX, 42)
        return float(ch.Arrayf32(ch.mean(ch.max(f32(100) * ch.exp(
            f32(0.03) + f32(0.2) * ch.rng_normal_make(g, 2048, 2048)) - f32(100), f32(0)))).read_scalar())
    ref = payoff()
    saved = ch._vm
    dev = ch.Device(config="ReduceAccum=f32")
    try:
        ch._vm = dev
        got = payoff()
    finally:
        ch._vm = saved
        dev.close()
    assert got != 0.0 and abs(got - ref) <= 1e-6 * abs(ref), (got, ref)


def test_reduction_vectorised_slots(ch):
    """make2 with a list of host arrays: one trace, `slots` independent sums."""
    rng = np.random.default_rng(2)
    data = rng.standard_normal((6, 33, 65)).astype(np.float32)
    A = ch.make2(data)
    got = ch.Arrayf64(ch.sum(ch.convert_f64(A))).read_scalar()
    want = data.astype(np.float64).reshape(6, -1).sum(axis=1)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-9)


def test_matmul_sum_trace_simt(ch):
    """C = matmul(A, B); s = sum(C * C) (the 512x512 trace) through the FP32
    CUDA-core GEMM, against the FP64 oracle."""
    n = 256
    A = oracle.rng_fill(n * n, seed=0, limits=(-1.0, 1.0)).reshape(n, n)
    B = oracle.rng_fill(n * n, seed=n * n, limits=(-1.0, 1.0)).reshape(n, n)
    dev_cfg = ch.vm()
    a, b = ch.make2(A), ch.make2(B)
    c = ch.Arrayf32(ch.matmul(a, b))
    s = ch.Arrayf32(ch.sum(c * c))
    Cg = c.read2()
    sg = float(s.read_scalar())
    C64 = oracle.gemm_f64(A, B)
    bound = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    # bf16x3 default (split-precision) or fp32: normalised error <= 2^-14
    assert np.max(np.abs(Cg - C64) / bound) <= 2.0 ** -14
    s64 = float((Cg.astype(np.float64) ** 2).sum())
    assert abs(sg - s64) <= 1e-6 * s64
    del dev_cfg


def test_gemv_trace(ch):
    rng = np.random.default_rng(3)
    for (m, n) in ((300, 517), (64, 64)):
        A = rng.uniform(-1, 1, (m, n)).astype(np.float32)
        x = rng.uniform(-1, 1, n).astype(np.float32)
        y = ch.Arrayf32(ch.matmul(ch.make2(A), ch.make1(x))).read1()
        want = oracle.gemv_f64(A, x)
        assert np.max(np.abs(y - want)) <= 1e-5 * np.sqrt(n)
        yt = ch.Arrayf32(ch.matmul(ch.make1(rng.uniform(-1, 1, m).astype(np.float32)), ch.make2(A))).read1()
        assert yt.shape == (n,)


def test_gemv_f64(ch):
    rng = np.random.default_rng(4)
    A = rng.uniform(-1, 1, (257, 130))
    x = rng.uniform(-1, 1, 130)
    y = ch.Arrayf64(ch.matmul(ch.make2(A), ch.make1(x))).read1()
    assert np.max(np.abs(y - A @ x)) <= 1e-13


def test_transpose(ch):
    a = np.arange(35 * 17, dtype=np.float32).reshape(17, 35)
    t = ch.Arrayf32(ch.transpose(ch.make2(a))).read2()
    assert np.array_equal(t, a.T)


def test_gather2_floor_wrap_bit_exact(ch):
    rng = np.random.default_rng(5)
    H, W = 24, 40
    A = rng.uniform(0, 1, (H, W)).astype(np.float32)
    X = rng.uniform(-W, 2 * W, (H, W)).astype(np.float32)
    Y = rng.uniform(-H, 2 * H, (H, W)).astype(np.float32)
    got = ch.Arrayf32(ch.gather2_floor(ch.make2(A), ch.make2(X), ch.make2(Y))).read2()
    assert np.array_equal(got, oracle.gather2_floor(A, X, Y))


def kirsch_expr(ch, A, W, H):
    X, Y = ch.index_f32(0, W, H), ch.index_f32(1, W, H)
    one = f32(1)
    n = [ch.gather2_floor(A, X - one, Y - one), ch.gather2_floor(A, X, Y - one), ch.gather2_floor(A, X + one, Y - one),
         ch.gather2_floor(A, X + one, Y), ch.gather2_floor(A, X + one, Y + one), ch.gather2_floor(A, X, Y + one),
         ch.gather2_floor(A, X - one, Y + one), ch.gather2_floor(A, X - one, Y)]
    total = n[0] + n[1] + n[2] + n[3] + n[4] + n[5] + n[6] + n[7]
    r = [f32(8) * ((n[k] + n[(k + 1) % 8]) + n[(k + 2) % 8]) - f32(3) * total for k in range(8)]
    return ch.max(ch.max(ch.max(r[0], r[1]), ch.max(r[2], r[3])), ch.max(ch.max(r[4], r[5]), ch.max(r[6], r[7])))


def test_kirsch_trace_bit_exact(ch):
    H, W = 96, 128
    img = oracle.rng_fill(W * H, seed=5).reshape(H, W)
    A = ch.make2(img)
    got = ch.Arrayf32(kirsch_expr(ch, A, W, H)).read2()
    assert np.array_equal(got, oracle.kirsch(img))


def _kirsch_tree_numpy(img):
    """The traced Kirsch program in numpy (the image's precision), one IEEE
    operation at a time: periodic neighbours, 8 * ((n_k + n_k+1) + n_k+2) -
    3 * total, and the max tree of chai's `a < b ? b : a`."""
    f = img.dtype.type
    n = [np.roll(np.roll(img, -dy, 0), -dx, 1) for dx, dy in
         ((-1, -1), (0, -1), (1, -1), (1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0))]
    with np.errstate(all="ignore"):
        total = n[0]
        for k in range(1, 8):
            total = total + n[k]
        t3 = f(3) * total
        r = [f(8) * ((n[k] + n[(k + 1) % 8]) + n[(k + 2) % 8]) - t3 for k in range(8)]
    mx = lambda a, b: np.where(a < b, b, a)
    return mx(mx(mx(r[0], r[1]), mx(r[2], r[3])), mx(mx(r[4], r[5]), mx(r[6], r[7])))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_max_affine_fusion_is_exact_on_special_values(ch, dt):
    """The max-of-affine rewrite (c * max(s_k) - t for a max tree of
    c * s_k - t, FuseMaxAffine; f32 trees through max.NaN) against the plain
    tree (FuseMaxAffine=0) and a numpy restatement, on an image with signed
    zeros, NaNs, infinities, subnormals and values whose 8 * s overflows:
    bit-identical on the GPU, and equal to numpy except for the sign of NaNs
    (parity exception 7)."""
    H, W = 64, 64
    big = 3e38 if dt == np.float32 else 1.7e308
    rng = np.random.default_rng(21)
    img = rng.uniform(0, 1, (H, W)).astype(dt)
    img[8:16, 8:16] = np.where(rng.uniform(size=(8, 8)) < 0.5, dt(-0.0), dt(0.0))
    img[10, 40] = np.nan
    img[30, 5] = np.inf
    img[50, 50] = -np.inf
    img[40:43, 20:23] = dt(big)
    img[20:22, 55:58] = dt(-big)
    img[60, 1] = dt(1e-40 if dt == np.float32 else 1e-310)     # a subnormal
    arr = ch.Arrayf32 if dt == np.float32 else ch.Arrayf64
    ut = np.uint32 if dt == np.float32 else np.uint64
    outs = []
    for cfg in ("", "FuseMaxAffine=0"):
        saved = ch._vm
        dev = ch.Device(config=cfg) if cfg else None
        try:
            if dev:
                ch._vm = dev
            outs.append(arr(kirsch_expr(ch, ch.make2(img), W, H)).read2())
        finally:
            ch._vm = saved
            if dev:
                dev.close()
    fused, plain = outs
    assert fused.dtype == dt
    assert np.array_equal(fused.view(ut), plain.view(ut))
    want = _kirsch_tree_numpy(img)
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(fused), nan)
    assert np.array_equal(fused[~nan].view(ut), want[~nan].view(ut))
    assert (fused == 0).any() and np.isinf(fused).any() and nan.any()


@pytest.mark.parametrize("shape", [(96, 128), (130, 517), (16, 16), (300, 1024)])
def test_stencil_tiles_bit_exact(ch, shape):
    """Constant-offset gathers run as 2-D shared-memory tiles (TMA for
    interior tiles when W % 4 == 0, wrapped loads at borders and otherwise);
    the periodic wrap must match the interpreter exactly at every border."""
    H, W = shape
    rng = np.random.default_rng(W + H)
    img = rng.standard_normal((H, W)).astype(np.float32)
    A = ch.make2(img)
    X, Y = ch.index_f32(0, W, H), ch.index_f32(1, W, H)
    e = (ch.gather2_floor(A, X + f32(2), Y - f32(1)) * f32(3) - ch.gather2_floor(A, X - f32(1), Y + f32(3))
         + ch.gather1_floor(A, X + f32(4)))
    got = ch.Arrayf32(e).read2()
    roll = lambda dx, dy: np.roll(np.roll(img, -dy, axis=0), -dx, axis=1)
    want = roll(2, -1) * f32(3) - roll(-1, 3) + roll(4, 0)
    assert np.array_equal(got, want)


def test_stencil_with_reduction(ch):
    H, W = 256, 512
    img = oracle.rng_fill(W * H, seed=9).reshape(H, W)
    A = ch.make2(img)
    X, Y = ch.index_f32(0, W, H), ch.index_f32(1, W, H)
    s = float(ch.Arrayf64(ch.sum(ch.convert_f64(ch.gather2_floor(A, X + f32(1), Y) - A))).read_scalar())
    want = (np.roll(img, -1, axis=1).astype(np.float32) - img).astype(np.float64).sum()
    assert abs(s - want) <= 1e-9 * max(1.0, np.abs(img).sum())


def test_c1_trace_with_generated_inputs(ch):
    """C1 as the bench runs it: A and B filled inside the trace by one chai
    Philox generator (seed 0; the second fill starts 512*512 counters later),
    C = matmul(A, B), s = sum(C * C).  The inputs are bit-exact against the
    oracle's fills; s within 1e-4 relative of the FP64 product's (bf16x3
    products: normalised element error <= 2^-14)."""
    import bench
    n = bench.C1_N
    g = ch.RNGf32(ch.RNG_PHILOX, 0)
    a = ch.Arrayf32(ch.rng_uniform_make(g, n, n, 1, -1.0, 1.0))
    b = ch.Arrayf32(ch.rng_uniform_make(g, n, n, 1, -1.0, 1.0))
    c = ch.Arrayf32(ch.matmul(a, b))
    s = ch.Arrayf32(ch.sum(c * c))
    A = oracle.rng_fill(n * n, seed=0, limits=(-1.0, 1.0)).reshape(n, n)
    B = oracle.rng_fill(n * n, seed=n * n, limits=(-1.0, 1.0)).reshape(n, n)
    assert np.array_equal(a.read2(), A) and np.array_equal(b.read2(), B)
    C64 = A.astype(np.float64) @ B.astype(np.float64)
    s64 = float((C64 ** 2).sum())
    assert abs(float(s.read_scalar()) - s64) <= 1e-4 * s64
