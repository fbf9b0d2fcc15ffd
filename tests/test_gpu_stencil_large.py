"""Stencil tiles on images of many tiles: interior tiles staged by TMA,
border tiles by TMA with the elements outside the image replaced by wrapped
loads (or, StencilBorderTma=0, entirely by wrapped loads: the periodic wrap
of interp/InterpGather.hpp:31-44 without a division for coordinates within
one period), ragged last tile rows and columns, f64 and two-source stencils,
for several tile heights, register limits and packing options.  Bit-exact
against the oracle's Kirsch and numpy rolls."""
import ctypes as C

import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32

CONFIGS = ["", "StencilRows=16", "StencilRows=8", "StencilRows=64", "StencilMinBlocks=5", "PackF32=0",
           "PackF32Stencil=1", "StencilBorderTma=0", "StencilBorderTma=0 StencilRows=16"]


def _eval_on(ch, dev, imgs, expr):
    """Record expr(*inputs) over input variables bound to fresh buffers and
    evaluate it on `dev`; return the result image."""
    H, W = imgs[0].shape
    ch._Client.pending, saved = [], ch._Client.pending
    try:
        ins = []
        for img in imgs:
            prec = L.F64 if img.dtype == np.float64 else L.F32
            var = next(ch._Client.vars)
            ins.append((var, prec, ch._Raw([ch._bc(L.BC_VARIABLE, var, 0)], prec, W, H)))
        out = expr(*[x[2] for x in ins])
        stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    finally:
        ch._Client.pending = saved
    binds, ids = [], []
    for k, (img, (var, prec, _)) in enumerate(zip(imgs, ins)):
        bid = 7700 + k
        L.check(L.lib().chai_cuda_buffer_alloc(dev.ctx, bid, img.nbytes), dev.ctx)
        L.check(L.lib().chai_cuda_upload(dev.ctx, bid, img.ctypes.data_as(C.c_void_p), img.nbytes), dev.ctx)
        binds.append((var, prec, W, H, 1, 0, bid))
        ids.append(bid)
    binds.append((out.var, out.prec, W, H, 1, 0, 7799))
    ids.append(7799)
    dev.evaluate(stmts, binds)
    got = dev.readback(7799, W * H, np.float64 if out.prec == L.F64 else np.float32).reshape(H, W)
    for i in ids:
        dev.release(i)
    return got


@pytest.fixture(scope="module", params=CONFIGS)
def cdev(chai_dev, request):
    import chai_b200.api as ch
    dev = ch.Device(config=request.param or None)
    yield dev
    dev.close()


def _roll(img, dx, dy):
    return np.roll(np.roll(img, -dy, axis=0), -dx, axis=1)


@pytest.mark.parametrize("shape", [(2048, 4096), (1000, 2052)])
def test_kirsch_many_tiles(cdev, shape):
    """8 gathers of one f32 source; (1000, 2052): ragged last tile row and
    column, W % 4 == 0 so interior tiles use TMA."""
    import chai_b200.api as ch
    from tests.test_gpu_trace import kirsch_expr
    H, W = shape
    img = oracle.rng_fill(W * H, seed=H + W).reshape(H, W)
    got = _eval_on(ch, cdev, [img], lambda A: ch.Arrayf32(kirsch_expr(ch, A, W, H)))
    assert np.array_equal(got, oracle.kirsch(img))


def test_f64_source_many_tiles(cdev):
    """An f64 source (8-byte elements, 16-byte shared windows of 2 values);
    W % 4 != 0 keeps every tile on the wrapped-load path."""
    import chai_b200.api as ch
    H, W = 700, 1030
    img = np.random.default_rng(3).standard_normal((H, W))
    X, Y = (lambda: ch.index_f64(0, W, H)), (lambda: ch.index_f64(1, W, H))
    got = _eval_on(ch, cdev, [img], lambda A: ch.Arrayf64(
        ch.gather2_floor(A, X() + 2.0, Y() - 3.0) * 0.5 - ch.gather2_floor(A, X() - 1.0, Y() + 1.0)))
    assert np.array_equal(got, _roll(img, 2, -3) * 0.5 - _roll(img, -1, 1))


def test_two_sources_many_tiles(cdev):
    """Two f32 sources in one stencil (two staged tiles per CTA)."""
    import chai_b200.api as ch
    H, W = 1536, 2048
    rng = np.random.default_rng(4)
    a = rng.standard_normal((H, W)).astype(f32)
    b = rng.standard_normal((H, W)).astype(f32)
    X, Y = (lambda: ch.index_f32(0, W, H)), (lambda: ch.index_f32(1, W, H))
    got = _eval_on(ch, cdev, [a, b], lambda A, B: ch.Arrayf32(
        ch.gather2_floor(A, X() + f32(1), Y() + f32(2)) - ch.gather2_floor(B, X() - f32(3), Y() - f32(1)) * f32(2)))
    assert np.array_equal(got, _roll(a, 1, 2) - _roll(b, -3, -1) * f32(2))
