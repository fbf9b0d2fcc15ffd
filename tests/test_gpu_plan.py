"""Plan cache: a trace evaluated again with the same structure (cells,
scalars, shapes, bindings) but different buffers and contents is replayed
from the recorded device operations; results must equal a fresh translation
and the oracle.  A change of any scalar (e.g. an RNG seed) is a new trace."""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.fixture
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


def replays(dev):
    n = C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(dev.ctx, b"plan_replay", None, C.byref(n), 0), dev.ctx)
    return n.value


def test_kirsch_replay_with_new_image(ch, chai_dev):
    from tests.test_gpu_trace import kirsch_expr
    H, W = 64, 96
    outs = []
    r0 = replays(chai_dev)
    for seed in (5, 6, 7):
        img = oracle.rng_fill(W * H, seed=seed).reshape(H, W)
        got = ch.Arrayf32(kirsch_expr(ch, ch.make2(img), W, H)).read2()
        assert np.array_equal(got, oracle.kirsch(img))
        outs.append(got)
    assert replays(chai_dev) - r0 == 2
    assert not np.array_equal(outs[0], outs[1])


def test_matmul_sum_replay(ch, chai_dev):
    n = 128
    r0 = replays(chai_dev)
    for seed in (1, 2):
        rng = np.random.default_rng(seed)
        A = rng.uniform(-1, 1, (n, n)).astype(f32)
        B = rng.uniform(-1, 1, (n, n)).astype(f32)
        c = ch.Arrayf32(ch.matmul(ch.make2(A), ch.make2(B)))
        s = ch.Arrayf32(ch.sum(c * c))
        Cg = c.read2()
        sg = float(s.read_scalar())
        C64 = oracle.gemm_f64(A, B)
        bound = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
        assert np.max(np.abs(Cg - C64) / bound) <= 2.0 ** -14
        assert abs(sg - float((Cg.astype(np.float64) ** 2).sum())) <= 1e-6 * sg
    assert replays(chai_dev) - r0 >= 1


def test_rng_reduction_replay_and_new_seed(ch, chai_dev):
    W, H = 256, 64

    def payoff(seed):
        g = ch.RNGf32(ch.RNG_PHILOX, seed)
        z = ch.rng_normal_make(g, W, H)
        return float(ch.Arrayf32(ch.mean(ch.max(f32(100) * ch.exp(f32(0.03) + f32(0.2) * z) - f32(100),
                                                f32(0)))).read_scalar())
    r0 = replays(chai_dev)
    a, b = payoff(42), payoff(42)
    assert a == b
    assert replays(chai_dev) - r0 == 1
    c = payoff(43)
    assert replays(chai_dev) - r0 == 1            # a new seed is a new trace
    z = oracle.rng_fill(W * H, dist=1, seed=43).astype(f32)
    want = np.maximum(f32(100) * np.exp(f32(0.03) + f32(0.2) * z) - f32(100), f32(0)).astype(np.float64).mean()
    assert abs(c - want) <= 1e-5 * abs(want)


def _kirsch_on(ch, dev, img, in_id, out_id):
    """Record the Kirsch trace over an input variable bound to buffer in_id and
    evaluate it on `dev` (a context of its own) into buffer out_id."""
    from tests.test_gpu_trace import kirsch_expr
    H, W = img.shape
    ch._Client.pending, saved = [], ch._Client.pending
    try:
        a_var = next(ch._Client.vars)
        A = ch._Raw([ch._bc(L.BC_VARIABLE, a_var, 0)], 4, W, H)
        K = ch.Arrayf32(kirsch_expr(ch, A, W, H))
        stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    finally:
        ch._Client.pending = saved
    L.check(L.lib().chai_cuda_buffer_alloc(dev.ctx, in_id, img.nbytes), dev.ctx)
    L.check(L.lib().chai_cuda_upload(dev.ctx, in_id, img.ctypes.data_as(C.c_void_p), img.nbytes), dev.ctx)
    dev.evaluate(stmts, [(a_var, 4, W, H, 1, 0, in_id), (K.var, 4, W, H, 1, 0, out_id)])
    out = dev.readback(out_id, W * H, np.float32).reshape(H, W)
    for i in (in_id, out_id):
        dev.release(i)
    return out


@pytest.mark.parametrize("cache", [0, 1])
def test_plan_cache_on_and_off_agree(ch, cache):
    dev = ch.Device(config="PlanCache=%d" % cache)
    try:
        for k, seed in enumerate((9, 10, 11)):
            img = oracle.rng_fill(32 * 48, seed=seed).reshape(32, 48)
            got = _kirsch_on(ch, dev, img, 500 + 2 * k, 501 + 2 * k)
            assert np.array_equal(got, oracle.kirsch(img))
        assert replays(dev) == (2 if cache else 0)
    finally:
        dev.close()


def graph_launches(dev):
    n = C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(dev.ctx, b"plan_graph", None, C.byref(n), 0), dev.ctx)
    return n.value


def _c1_on(ch, dev, seed, out_id):
    """The C1 trace (Philox fills, 512^3 matmul on the tensor cores, sum(C*C))
    evaluated on `dev` into buffer out_id: RNG kernels, the split prepass, the
    GEMM (context scratch), a fused reduction and its combine (temporaries)."""
    import bench
    ch._Client.pending, saved = [], ch._Client.pending
    try:
        s = ch.Arrayf32(bench.c1_expr(ch, ch.RNGf32(ch.RNG_PHILOX, seed), 256))
        stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    finally:
        ch._Client.pending = saved
    dev.evaluate(stmts, [(s.var, 4, 1, 1, 1, 0, out_id)])
    return float(dev.readback(out_id, 1, np.float32)[0])


def test_graph_replay_c1_and_kirsch(ch):
    """PlanGraph=1: the third and later evaluations of a repeated trace run as
    one captured CUDA graph (plan_graph counter); results equal the plain
    replay's (PlanGraph=0) bit for bit, and the graph is captured again when
    the trace's buffers move (new buffer ids)."""
    g, p = ch.Device(config="PlanGraph=1"), ch.Device(config="PlanGraph=0")
    try:
        want = [_c1_on(ch, p, 3, 700) for _ in range(3)]
        got = [_c1_on(ch, g, 3, 700) for _ in range(4)]
        assert len(set(want)) == 1 and all(x == want[0] for x in got), (got, want)
        assert graph_launches(g) >= 2 and graph_launches(p) == 0
        n0 = graph_launches(g)
        # Kirsch over fixed buffers 900 -> 901, new image contents each time
        from tests.test_gpu_trace import kirsch_expr
        H, W = 40, 64
        ch._Client.pending, saved = [], ch._Client.pending
        try:
            a_var = next(ch._Client.vars)
            A = ch._Raw([ch._bc(L.BC_VARIABLE, a_var, 0)], 4, W, H)
            K = ch.Arrayf32(kirsch_expr(ch, A, W, H))
            stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
        finally:
            ch._Client.pending = saved
        for seed in (9, 10, 11, 12):
            img = oracle.rng_fill(W * H, seed=seed).reshape(H, W)
            L.check(L.lib().chai_cuda_upload(g.ctx, 900, img.ctypes.data_as(C.c_void_p), img.nbytes), g.ctx)
            g.evaluate(stmts, [(a_var, 4, W, H, 1, 0, 900), (K.var, 4, W, H, 1, 0, 901)])
            out = g.readback(901, W * H, np.float32).reshape(H, W)
            assert np.array_equal(out, oracle.kirsch(img)), seed
        assert graph_launches(g) - n0 >= 2
    finally:
        g.close()
        p.close()
