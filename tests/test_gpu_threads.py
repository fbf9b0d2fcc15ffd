"""Read-back and release from client threads while the device thread
evaluates (memmgr/MemTrans.hpp:43-47 guards the reference's device memory
with _memMutex for the same reason: client threads call swizzle and
untrackMem, common/MemCallback.hpp:13-21, while the device thread runs a
trace).  One thread evaluates an element trace over its own buffers again and
again; three threads read back and then release disjoint sets of other
buffers.  Every read-back must return the uploaded bytes, every release must
succeed once, a released id must then be unknown, and every evaluation must
give the right result."""
import ctypes as C
import threading

import numpy as np
import pytest

from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu
f32 = np.float32


def test_readback_and_release_during_evaluate(chai_dev):
    import chai_b200.api as ch
    dev = ch.Device()
    lib = L.lib()
    try:
        # buffers the client threads own: 3 threads x 40 buffers
        data = {}
        for t in range(3):
            for k in range(40):
                bid = 1000 + 100 * t + k
                arr = np.full(4096 + 37 * k, t * 1000 + k, dtype=np.float32)
                L.check(lib.chai_cuda_upload(dev.ctx, bid, arr.ctypes.data_as(C.c_void_p), arr.nbytes), dev.ctx)
                data[bid] = arr
        # the device thread's trace: Y = 2 X + 1 over a bound input
        W, H = 1024, 512
        x = np.random.default_rng(1).standard_normal((H, W)).astype(f32)
        L.check(lib.chai_cuda_upload(dev.ctx, 1, x.ctypes.data_as(C.c_void_p), x.nbytes), dev.ctx)
        saved = ch._Client.pending
        ch._Client.pending = []
        try:
            xv = next(ch._Client.vars)
            X = ch._Raw([ch._bc(L.BC_VARIABLE, xv, 0)], L.F32, W, H)
            Y = ch.Arrayf32(f32(2) * X + f32(1))
            stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
        finally:
            ch._Client.pending = saved
        binds = [(xv, L.F32, W, H, 1, 0, 1), (Y.var, L.F32, W, H, 1, 0, 2)]
        errors = []
        stop = threading.Event()

        def evaluator():
            try:
                for _ in range(200):
                    dev.evaluate(stmts, binds)
                    if stop.is_set():
                        break
            except Exception as e:           # noqa: BLE001 -- reported below
                errors.append(("evaluate", repr(e)))

        def client(t):
            try:
                ids = [1000 + 100 * t + k for k in range(40)]
                for rep in range(5):
                    for bid in ids:
                        out = np.empty_like(data[bid])
                        st = lib.chai_cuda_readback(dev.ctx, bid, out.ctypes.data_as(C.c_void_p), out.nbytes)
                        if st != 0 or not np.array_equal(out, data[bid]):
                            errors.append(("readback", bid, st))
                for bid in ids:
                    if lib.chai_cuda_release(dev.ctx, bid) != 0:
                        errors.append(("release", bid))
                    out = np.empty(4, dtype=np.float32)
                    if lib.chai_cuda_readback(dev.ctx, bid, out.ctypes.data_as(C.c_void_p), 16) != -6:
                        errors.append(("released id still known", bid))
            except Exception as e:           # noqa: BLE001
                errors.append(("client", t, repr(e)))

        threads = [threading.Thread(target=evaluator)] + [threading.Thread(target=client, args=(t,)) for t in range(3)]
        for th in threads:
            th.start()
        for th in threads[1:]:
            th.join(timeout=300)
        stop.set()
        threads[0].join(timeout=300)
        assert not any(th.is_alive() for th in threads)
        assert not errors, errors[:5]
        got = dev.readback(2, W * H, np.float32).reshape(H, W)
        assert np.array_equal(got, f32(2) * x + f32(1))
    finally:
        dev.close()
