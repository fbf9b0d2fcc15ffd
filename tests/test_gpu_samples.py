"""The reference's own sample programs (sample/*.cpp), written against the
front-end mirror exactly as they are written against api/chai.h, run end to
end on the GPU:

  md5.cpp      64 rounds of MD5 over 20 messages as one u32 trace (rotate,
               and / or / xor / not, u32 literals), checked against hashlib;
  cg.cpp       conjugate gradient: matrix-vector products, dot_product results
               broadcast as 1x1 arrays, one trace per iteration (each reads
               the residual norm), checked against numpy.linalg.solve;
  loopsum.cpp  A = A + mean(B) in nested loops, B += 1, sum(A): exact.
"""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
u32 = np.uint32
f32 = np.float32


@pytest.fixture
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


R = [7, 12, 17, 22] * 4 + [5, 9, 14, 20] * 4 + [4, 11, 16, 23] * 4 + [6, 10, 15, 21] * 4
K = [int(abs(np.sin(i + 1)) * 2 ** 32) & 0xffffffff for i in range(64)]
H = (0x67452301, 0xefcdab89, 0x98badcfe, 0x10325476)


def _md5_words(msg: bytes):
    pad = msg + b"\x80" + b"\x00" * ((55 - len(msg)) % 64) + (8 * len(msg)).to_bytes(8, "little")
    assert len(pad) == 64
    return np.frombuffer(pad, dtype="<u4").astype(np.uint32)


def test_md5_sample(ch):
    texts = [("cleartext message number %d" % i).encode() for i in range(20)]
    W = np.stack([_md5_words(t) for t in texts], axis=1)       # 16 x N, word-major as the sample lays it out
    N = len(texts)
    w = [ch.make1(np.ascontiguousarray(W[j])) for j in range(16)]
    a = ch.Arrayu32(u32(H[0]) * ch.ones_u32(N))
    b = ch.Arrayu32(u32(H[1]) * ch.ones_u32(N))
    c = ch.Arrayu32(u32(H[2]) * ch.ones_u32(N))
    d = ch.Arrayu32(u32(H[3]) * ch.ones_u32(N))
    for j in range(64):
        if j <= 15:
            f, g = (b & c) | ((~b) & d), j
        elif j <= 31:
            f, g = (d & b) | ((~d) & c), (5 * j + 1) % 16
        elif j <= 47:
            f, g = b ^ c ^ d, (3 * j + 5) % 16
        else:
            f, g = c ^ (b | (~d)), (7 * j) % 16
        f = ch.Arrayu32(f)
        temp = d
        d = c
        c = b
        b = ch.Arrayu32(b + ch.rotate(a + f + u32(K[j]) + w[g], u32(R[j])))
        a = temp
    outs = [x.read1() for x in (a, b, c, d)]
    for i, t in enumerate(texts):
        digest = b"".join(int((H[k] + int(outs[k][i])) & 0xffffffff).to_bytes(4, "little") for k in range(4))
        assert digest.hex() == hashlib.md5(t).hexdigest()


@pytest.mark.parametrize("N", [20, 96])
def test_conjugate_gradient_sample(ch, N):
    rng = np.random.default_rng(N)
    M = rng.uniform(0, 1, (N, N)).astype(f32)
    cpuA = (M @ M.T / N + np.eye(N, dtype=f32)).astype(f32)   # symmetric positive definite
    cpub = rng.uniform(0, 1, N).astype(f32)
    x = ch.Arrayf32(ch.zeros_f32(N))
    A = ch.make2(cpuA)
    bb = ch.make1(cpub)
    residuals = ch.Arrayf32(bb - ch.matmul(A, x))
    p = ch.Arrayf32(residuals)
    newRR = ch.Arrayf32(ch.dot_product(residuals, residuals))
    for it in range(N):
        oldRR = newRR
        Ap = ch.Arrayf32(ch.matmul(A, p))
        dp = ch.Arrayf32(ch.dot_product(p, Ap))
        newX = ch.Arrayf32(x + p * oldRR / dp)
        newResiduals = ch.Arrayf32(residuals - Ap * oldRR / dp)
        newRR = ch.Arrayf32(ch.dot_product(newResiduals, newResiduals))
        newP = ch.Arrayf32(newResiduals + p * newRR / oldRR)
        p = newP
        residuals = newResiduals
        if float(oldRR.read_scalar()) <= 1e-10:
            break
        x = newX
    got = x.read1()
    want = np.linalg.solve(cpuA.astype(np.float64), cpub.astype(np.float64))
    assert np.max(np.abs(got - want)) <= 1e-3 * np.max(np.abs(want)), (it, got[:4], want[:4])


def test_loopsum_sample(ch):
    rng = np.random.default_rng(10)
    data = rng.uniform(0, 1, (10, 100)).astype(f32)
    for i in range(10):
        A = ch.make1(data[i])
        B = ch.Arrayf32(f32(5) * ch.ones_f32(1))
        for j in range(2):
            for k in range(3):
                A = ch.Arrayf32(A + ch.mean(B))
            B = ch.Arrayf32(B + f32(1))
        got = float(ch.Arrayf32(ch.sum(A)).read_scalar())
        want = data[i].copy()
        for j in range(2):
            for k in range(3):
                want = want + f32(5 + j)
        assert abs(got - float(want.astype(np.float64).sum())) <= 1e-5 * abs(got)


def test_pi_sample(ch):
    """sample/pi.cpp: two uniform fills from one generator (the second starts
    where the first ended), sqrt(X^2 + Y^2) <= 1, 4 sum / NSET; exact."""
    import oracle
    NSET = 1000000
    G = ch.RNGf32(ch.RNG_DEFAULT, 271828)
    X = ch.Arrayf32(ch.rng_uniform_make(G, NSET, 1, 1, 0.0, 1.0))
    Y = ch.Arrayf32(ch.rng_uniform_make(G, NSET, 1, 1, 0.0, 1.0))
    distance_from_zero = ch.Arrayf32(ch.sqrt(X * X + Y * Y))
    inside_circle = ch.Arrayf32(distance_from_zero <= f32(1.0))
    pi = float(ch.Arrayf32(f32(4.0) * ch.sum(inside_circle) / NSET).read_scalar())
    x = oracle.rng_fill(NSET, seed=271828, limits=(0.0, 1.0))
    y = oracle.rng_fill(NSET, seed=271828 + NSET, limits=(0.0, 1.0))
    count = f32(np.count_nonzero(np.sqrt(x * x + y * y) <= f32(1.0)))
    assert pi == float(f32(f32(4.0) * count) / f32(NSET))
    assert abs(pi - np.pi) < 0.01


def test_american_option_sample(ch):
    """sample/finance/american_option.cpp: binomial tree in f64, one trace per
    step with a shrinking length, gather1_floor(option, IDX + 1) wrapping at
    the end; exact against the same arithmetic in numpy."""
    price, strike, vol, rate, maturity, steps = 100.0, 100.0, 0.25, 0.10, 1.0, 100
    R = np.exp(rate * (maturity / steps))
    up = np.exp(vol * np.sqrt(maturity / steps))
    down = 1.0 / up
    prUp = (R - down) / (up - down)
    prDown = 1.0 - prUp
    prices0 = np.empty(steps + 1)
    prices0[0] = price * down ** steps
    for i in range(1, steps + 1):
        prices0[i] = prices0[i - 1] * up * up
    option0 = np.maximum(prices0 - strike, 0.0)
    pg, og = prices0.copy(), option0.copy()
    pn, on = prices0.copy(), option0.copy()
    disc = float(np.exp(rate * (maturity / steps)))
    for i in range(steps):
        N = steps + 1 - i
        prices = ch.make1(pg[:N].copy())
        option = ch.make1(og[:N].copy())
        IDX = ch.index_f64(0, N)
        no_exercise = ch.Arrayf64((float(prDown) * ch.gather1_floor(option, IDX)
                                   + float(prUp) * ch.gather1_floor(option, IDX + 1)) / disc)
        prices = ch.Arrayf64(float(up) * prices)
        option = ch.Arrayf64(ch.max(no_exercise, prices - strike))
        pg[:N] = prices.read1()
        og[:N] = option.read1()
        # numpy, same operations and order
        o = on[:N]
        ne = (float(prDown) * o + float(prUp) * np.roll(o, -1)) / disc
        pn[:N] = float(up) * pn[:N]
        b = pn[:N] - strike
        on[:N] = np.where(ne < b, b, ne)
    assert np.array_equal(og, on) and np.array_equal(pg, pn)
    assert 10.0 < og[0] < 20.0
