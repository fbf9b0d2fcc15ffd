"""Many uneven traces in one persistent launch under a CUDA graph
(chai_cuda_evaluate_many) against the oracle (the same payoff computed on the
oracle's normals, Random123/R123Philox.cpp restated in oracle/r123.c) and
against the same traces evaluated one at a time.

Tolerances: against the oracle 1e-5 relative (f32 exp on the device against
numpy's, averaged over each trace; an infinite payoff, from a u = 0 draw,
must be infinite on both sides); against the single-trace path two f32 ulps
(results are the reductions rounded to f32, as read_scalar returns them, and
the two paths add FP64 partials in different orders)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
f32 = np.float32


def mc(ch, seed, W, H=1):
    g = ch.RNGf32(ch.RNG_PHILOX, seed)
    return ch.Arrayf32(ch.mean(ch.max(f32(100) * ch.exp(f32(0.03) + f32(0.2) * ch.rng_normal_make(g, W, H))
                                      - f32(100), f32(0))))


def close(a, b):
    """Equal (including the +inf a u0 = 0 draw gives in the reference's
    Box-Muller) or within two f32 ulps."""
    return a == b or abs(a - b) <= 2 * np.spacing(np.float32(abs(b)))


def lengths(n, seed=7):
    rng = np.random.default_rng(seed)
    return [int(4 * round(2.0 ** u / 4)) for u in rng.uniform(12, 22, n)]


def oracle_payoff(seed, W):
    z = oracle.rng_fill(W, dist=1, seed=seed).astype(np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        s = f32(100) * np.exp(f32(0.03) + f32(0.2) * z)
        return float(np.float32(np.maximum(s - f32(100), f32(0)).astype(np.float64).mean()))


def test_many_uneven_mc_traces_match_oracle_and_single(chai_dev):
    import chai_b200.api as ch
    Ls = lengths(64)
    traces = [ch.record(lambda L=L, s=s: mc(ch, 1000 + s, L))[0] for s, L in enumerate(Ls)]
    got = ch.evaluate_many(traces)
    again = ch.evaluate_many(traces)          # graph replay
    assert np.array_equal(got, again)
    for s, L in enumerate(Ls):
        want = oracle_payoff(1000 + s, L)
        assert got[s] == want or abs(got[s] - want) <= 1e-5 * abs(want), (s, L, got[s], want)
    for s, L in enumerate(Ls[:8] + Ls[-4:]):
        idx = Ls.index(L)
        want = float(mc(ch, 1000 + idx, L).read_scalar())
        assert close(got[idx], want), (idx, got[idx], want)


def test_many_changes_lengths_between_calls(chai_dev):
    import chai_b200.api as ch
    a = [ch.record(lambda L=L: mc(ch, 5, L))[0] for L in (4096, 8192, 65536)]
    b = [ch.record(lambda L=L: mc(ch, 5, L))[0] for L in (1 << 20, 4096, 12)]
    ra, rb = ch.evaluate_many(a), ch.evaluate_many(b)
    for L, r in zip((1 << 20, 4096, 12), rb):
        assert close(r, float(mc(ch, 5, L).read_scalar()))
    assert ra[0] == rb[1]


def test_many_falls_back_for_other_programs(chai_dev):
    import chai_b200.api as ch
    x = np.arange(1000, dtype=np.float32)
    traces = [ch.record(lambda s=s: ch.Arrayf32(ch.sum(ch.make1(x * s))))[0] for s in (1, 2)]
    r = ch.evaluate_many(traces)
    assert np.allclose(r, [x.sum(), 2 * x.sum()])


def test_repeated_batch_reuses_parse_but_sees_changed_scalars(chai_dev):
    """A batch identical to the previous call's is launched without parsing
    again; a batch that differs only in one trace's seed is parsed again and
    that trace's result follows the new seed."""
    import chai_b200.api as ch
    Ls = [4096, 65536, 12288]
    a = [ch.record(lambda L=L, s=s: mc(ch, 300 + s, L))[0] for s, L in enumerate(Ls)]
    b = [ch.record(lambda L=L, s=s: mc(ch, (900 if s == 1 else 300 + s), L))[0] for s, L in enumerate(Ls)]
    ra = ch.evaluate_many(a)
    assert np.array_equal(ch.evaluate_many(a), ra)
    rb = ch.evaluate_many(b)
    assert rb[0] == ra[0] and rb[2] == ra[2] and rb[1] != ra[1]
    assert close(rb[1], float(mc(ch, 900, 65536).read_scalar()))
    assert np.array_equal(ch.evaluate_many(a), ra)
