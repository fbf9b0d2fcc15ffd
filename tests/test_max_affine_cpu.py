"""The max-of-affine rewrite the trace translator applies
(chai_b200/csrc/trace_emit.cpp): a tree of chai max ops (`a < b ? b : a`)
whose leaves are c * s_k - t, with one constant c >= 1 and one t, equals
c * m - t with m the same tree over the s_k whenever t is not infinite; for
f32 the kernel also takes m as the IEEE maximum (max.NaN) when t is finite
and non-zero and no s_k is NaN.  Checked here in numpy, one IEEE operation at
a time, on random values with signed zeros, infinities, NaNs, subnormals and
magnitudes where c * s overflows."""
import numpy as np
import pytest


def chai_max(a, b):
    return np.where(a < b, b, a)


def tree(vals):
    """The Kirsch-shaped tree: ((0,1),(2,3)),((4,5),(6,7))."""
    m = chai_max
    return m(m(m(vals[0], vals[1]), m(vals[2], vals[3])), m(m(vals[4], vals[5]), m(vals[6], vals[7])))


def special_values(rng, dt, n):
    f = np.finfo(dt)
    pool = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, f.max, -f.max, f.max / 8, -f.max / 8, f.tiny / 4,
                     -f.tiny / 4, 1.0, -1.0, 3.0, 0.5], dtype=dt)
    x = rng.standard_normal(n).astype(dt) * dt(10) ** rng.integers(-3, 4, n).astype(dt)
    pick = rng.uniform(size=n) < 0.35
    x[pick] = pool[rng.integers(0, len(pool), pick.sum())]
    return x


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("c", [1.0, 3.0, 8.0, 1.5])
def test_rewrite_is_bit_exact_when_t_is_finite(dt, c):
    rng = np.random.default_rng(5)
    n = 200_000
    s = [special_values(rng, dt, n) for _ in range(8)]
    t = special_values(rng, dt, n)
    c = dt(c)
    with np.errstate(all="ignore"):
        want = tree([c * sk - t for sk in s])
        short = c * tree(s) - t
        nan_max = np.maximum.reduce(s)               # IEEE maximum with NaN propagation
        fast_f32 = c * nan_max - t
    ut = np.uint32 if dt == np.float32 else np.uint64
    use = ~np.isinf(t)
    bits = lambda a: a.view(ut)
    nan_w, nan_s = np.isnan(want), np.isnan(short)
    # the short form: same NaN positions, same bits elsewhere (NaN payloads
    # are the GPU's canonical NaN on the device; numpy keeps x86's)
    assert np.array_equal(nan_w[use], nan_s[use])
    ok = use & ~nan_w
    assert np.array_equal(bits(want[ok]), bits(short[ok]))
    # the max.NaN form under its own conditions
    use2 = use & (t != 0) & ~np.isnan(nan_max)
    assert np.array_equal(np.isnan(want[use2]), np.isnan(fast_f32[use2]))
    ok2 = use2 & ~np.isnan(want)
    assert np.array_equal(bits(want[ok2]), bits(fast_f32[ok2]))
    # the cases the kernel sends to the original tree do occur here
    assert (~use).any() and (use & (t == 0)).any() and (use & np.isnan(nan_max)).any()


def test_infinite_t_breaks_the_short_form():
    """Why the kernel keeps the tree when t is infinite: inf - inf."""
    f = np.float32
    s = [f(1), f(np.inf)] + [f(0)] * 6
    t = f(np.inf)
    with np.errstate(all="ignore"):
        want = tree([f(8) * sk - t for sk in s])
        short = f(8) * tree(s) - t
    assert np.isneginf(want) and np.isnan(short)
