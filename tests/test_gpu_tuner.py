"""Learned tuner on the GPU: the MLP's forward and backward kernels against the
CPU oracle (oracle/mlp.py), training, every configuration of the search space
computing the right product, the sweep / learned / exhaustive modes, the tuning
DB and the crash journal (autotune/AutoTuneMemo.hpp:20-28).

Tolerances: the GPU network runs in FP32 with FP32 accumulation, the oracle in
FP64.  Loss and predictions agree to 1e-4 relative; every gradient entry agrees
to 1e-3 relative plus 1e-5 of the largest gradient entry."""
import ctypes as C

import numpy as np
import pytest

from chai_b200 import _lib as L
from chai_b200 import api as ch
from chai_b200 import tuner as T
from oracle import mlp as OM

pytestmark = pytest.mark.gpu


def _cfg(d, us=0.0):
    c = L.chai_gemm_cfg()
    for k, v in d.items():
        setattr(c, k, v)
    c.cluster_m = d.get("cluster_m", 1)
    c.cluster_n = d.get("cluster_n", 1)
    c.measured_us = us
    return c


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        gemv = bool(rng.uniform() < 0.3)
        m, n_, k = (int(x) for x in np.exp(rng.uniform(np.log(64), np.log(16384), 3)))
        key = T.key(m, n_, k, int(rng.choice([L.GEMM_FP32, L.GEMM_BF16])), gemv)
        space = OM.space(gemv)
        d = space[int(rng.integers(len(space)))]
        out.append((key, _cfg(d, float(np.exp(rng.uniform(1, 9))))))
    return out


def _x_y(samples):
    x = np.stack([T.features(k, c) for k, c in samples]).astype(np.float64)
    y = np.array([np.float32(np.log(max(c.measured_us, 1e-3))) for _, c in samples], dtype=np.float64)
    return x, y


def test_mlp_forward_and_gradients_match_oracle(chai_dev):
    ctx = chai_dev.ctx
    w = OM.init(11)
    w[-2:] = [4.0, 1.5]
    T.set_weights(ctx, w)
    np.testing.assert_array_equal(T.get_weights(ctx), w)
    samples = _samples(300, seed=2)
    x, y = _x_y(samples)
    pred = T.predict(ctx, samples)
    np.testing.assert_allclose(pred, OM.predict_log_us(w, x), rtol=1e-4, atol=1e-4)
    loss, g = T.gradients(ctx, samples)
    loss_ref, g_ref = OM.loss_and_grads(w, x, y)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    assert g.shape == g_ref.shape
    np.testing.assert_allclose(g, g_ref, rtol=1e-3, atol=1e-5 * np.abs(g_ref).max())


def test_mlp_training_fits_and_stays_consistent_with_oracle(chai_dev):
    ctx = chai_dev.ctx
    samples = _samples(512, seed=4)
    x, _ = _x_y(samples)
    # a smooth synthetic cost surface of the features
    y = 2.0 + 3.0 * x[:, 0] * x[:, 1] + 2.0 * x[:, 2] - 1.5 * x[:, 6] * x[:, 0] + np.sin(4 * x[:, 11])
    for (_, c), v in zip(samples, y):
        c.measured_us = float(np.exp(v))
    loss0 = T.train(ctx, samples, epochs=1, lr=1e-3, seed=5)
    loss = T.train(ctx, samples, epochs=1500, lr=1e-3, seed=5)
    assert loss < 0.05 * loss0 and loss < 0.02, (loss0, loss)
    w = T.get_weights(ctx)
    np.testing.assert_allclose(T.predict(ctx, samples), OM.predict_log_us(w, x), rtol=1e-4, atol=1e-4)


def _db_line(key, d):
    c = _cfg(d)
    return "BEST %d %d %d %d %d %d %d %d %d %d %d %d %d 1.0\n" % (
        key.m, key.n, key.k, key.precision, key.is_gemv, c.block_m, c.block_n, c.block_k, c.stages, c.vec_width,
        c.cluster_m, c.cluster_n, c.group_m)


@pytest.mark.parametrize("prec,bound", [(L.GEMM_BF16X3, 2.0 ** -14), (L.GEMM_BF16, 2.0 ** -7)])
@pytest.mark.parametrize("shape", [(300, 520, 200), (1024, 640, 384)])
def test_every_tuned_gemm_config_is_correct(chai_dev, tmp_path, prec, bound, shape):
    import torch
    M, N, K = shape
    rng = np.random.default_rng(8)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    C64 = A.astype(np.float64) @ B.astype(np.float64)
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    a, b = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    key = T.key(M, N, K, prec)
    for i, d in enumerate(OM.space(False)):
        db = tmp_path / ("db%d" % i)
        db.write_text(_db_line(key, d))
        L.check(L.lib().chai_cuda_tune_db_load(chai_dev.ctx, str(db).encode()), chai_dev.ctx)
        c = torch.full((M, N), float("nan"), device="cuda")
        desc = L.chai_gemm_desc(prec, 0, 0, 0, M, N, K, a.data_ptr(), K, b.data_ptr(), N, c.data_ptr(), N, 1.0, 0.0,
                                1, 0, 0, 0)
        L.check(L.lib().chai_cuda_gemm(chai_dev.ctx, C.byref(desc)), chai_dev.ctx)
        L.check(L.lib().chai_cuda_synchronize(chai_dev.ctx), chai_dev.ctx)
        err = np.max(np.abs(c.cpu().numpy().astype(np.float64) - C64) / scale)
        assert err <= bound, (d, err)


@pytest.mark.parametrize("prec", [L.F32, L.F64])
def test_every_tuned_gemv_config_is_correct(chai_dev, tmp_path, prec):
    import torch
    M, N = 1000, 777
    dt = np.float32 if prec == L.F32 else np.float64
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (M, N)).astype(dt)
    x = rng.uniform(-1, 1, N).astype(dt)
    y64 = A.astype(np.float64) @ x.astype(np.float64)
    scale = np.abs(A).astype(np.float64) @ np.abs(x).astype(np.float64)
    a, xv = torch.from_numpy(A).cuda(), torch.from_numpy(x).cuda()
    key = T.key(M, N, precision=L.GEMM_FP32 if prec == L.F32 else L.GEMM_FP64, is_gemv=True)
    for i, d in enumerate(OM.space(True)):
        db = tmp_path / ("db%d" % i)
        db.write_text(_db_line(key, d))
        L.check(L.lib().chai_cuda_tune_db_load(chai_dev.ctx, str(db).encode()), chai_dev.ctx)
        y = torch.full((M,), float("nan"), dtype=a.dtype, device="cuda")
        L.check(L.lib().chai_cuda_gemv(chai_dev.ctx, prec, 0, M, N, 1.0, a.data_ptr(), N, xv.data_ptr(), 0.0,
                                       y.data_ptr()), chai_dev.ctx)
        L.check(L.lib().chai_cuda_synchronize(chai_dev.ctx), chai_dev.ctx)
        err = np.max(np.abs(y.cpu().numpy().astype(np.float64) - y64) / scale)
        assert err <= (2.0 ** -16 if prec == L.F32 else 2.0 ** -45), (d, err)


def test_sweep_learned_and_exhaustive_modes(tmp_path):
    journal = tmp_path / "journal"
    dev = ch.Device(config="TuneJournal=%s TopK=2" % journal)
    try:
        ctx = dev.ctx
        k = T.key(512, 512, 512, L.GEMM_BF16X3)
        cfgs = T.sweep(ctx, k)
        assert len(cfgs) == T.GEMM_SPACE
        assert all(0 < c.measured_us < 1e6 for c in cfgs)
        assert len(T.sweep(ctx, T.key(2048, 1024, is_gemv=True, precision=L.GEMM_FP32))) == T.GEMV_SPACE
        best = T.tune(ctx, k, L.TUNE_EXHAUSTIVE)
        assert T.cfg_id(best) in {T.cfg_id(c) for c in cfgs}
        # learned mode without a trained model falls back to the sweep
        n0 = journal.read_text().count("TRY ")
        T.tune(ctx, T.key(384, 256, 128, L.GEMM_BF16), L.TUNE_LEARNED)
        assert journal.read_text().count("TRY ") - n0 == T.GEMM_SPACE
        # train on a few sweeps, then learned mode times only the top k
        train_keys = [T.key(m, n, kk, p) for (m, n, kk) in [(256, 256, 256), (1024, 256, 512), (128, 2048, 256),
                                                           (768, 768, 1024)] for p in (L.GEMM_FP32, L.GEMM_BF16)]
        data, _ = T.collect(ctx, train_keys)
        samples = [(kk, c) for kk, cs in data for c in cs]
        T.train(ctx, samples, epochs=500)
        n0 = journal.read_text().count("TRY ")
        pick = T.tune(ctx, T.key(640, 512, 384, L.GEMM_BF16), L.TUNE_LEARNED)
        assert journal.read_text().count("TRY ") - n0 == 2
        assert T.cfg_id(pick) in {T.cfg_id(_cfg(d)) for d in OM.space(False)}
        assert journal.read_text().count("TRY ") == journal.read_text().count("OK ")
    finally:
        dev.close()


def test_journal_skips_configuration_that_crashed(tmp_path):
    journal = tmp_path / "journal"
    k = T.key(512, 384, 256, L.GEMM_BF16)
    bad = OM.space(False)[0]
    c = _cfg(bad)
    line = "%d %d %d %d %d %d %d %d %d %d %d %d %d" % (k.m, k.n, k.k, k.precision, k.is_gemv, c.block_m, c.block_n,
                                                      c.block_k, c.stages, c.vec_width, 1, 1, c.group_m)
    journal.write_text("TRY " + line + "\n")
    dev = ch.Device(config="TuneJournal=%s" % journal)
    try:
        cfgs = T.sweep(dev.ctx, k)
        by = {T.cfg_id(x): x.measured_us for x in cfgs}
        assert by[T.cfg_id(c)] >= 1e29
        assert sum(v < 1e29 for v in by.values()) == T.GEMM_SPACE - 1
        assert T.cfg_id(T.tune(dev.ctx, k, L.TUNE_EXHAUSTIVE)) != T.cfg_id(c)
    finally:
        dev.close()


def test_tuning_db_and_weights_round_trip(tmp_path):
    db = tmp_path / "tune.db"
    dev = ch.Device()
    try:
        ctx = dev.ctx
        k = T.key(256, 768, 512, L.GEMM_BF16X3)
        best = T.tune(ctx, k, L.TUNE_EXHAUSTIVE)
        T.train(ctx, [(k, c) for c in T.sweep(ctx, k)], epochs=50)
        w = T.get_weights(ctx)
        L.check(L.lib().chai_cuda_tune_db_save(ctx, str(db).encode()), ctx)
    finally:
        dev.close()
    text = db.read_text()
    # the line holds the key and every field of the configuration the sweep
    # chose (one-CTA or CTA-pair tile, whichever timed best)
    assert text.startswith("BEST 256 768 512 %d 0 %d %d %d %d %d %d %d %d " % (
        L.GEMM_BF16X3, best.block_m, best.block_n, best.block_k, best.stages, best.vec_width, best.cluster_m,
        best.cluster_n, best.group_m))
    dev = ch.Device(config="TuneDB=%s" % db)
    try:
        np.testing.assert_array_equal(T.get_weights(dev.ctx), w)
    finally:
        dev.close()


def test_unsupported_tuning_keys_are_rejected(chai_dev):
    for k in (T.key(0, 64, 64), T.key(64, 64, 64, L.GEMM_FP8), T.key(64, 64, 64, L.GEMM_FP64)):
        out = L.chai_gemm_cfg()
        st = L.lib().chai_cuda_tune(chai_dev.ctx, C.byref(k), L.TUNE_EXHAUSTIVE, C.byref(out))
        assert st in (-1, -2)


def test_learned_tuner_gain_over_defaults_and_cold_start(tmp_path):
    """What the trained network gains over the method without it.  Exhaustive
    sweeps of 1000 training keys (M, N, K log-uniform in [64, 2048]; fp32 via
    bf16x3, bf16, and f32 GEMV) train the cost model on the GPU; on 40
    held-out keys of the same distribution the learned method (rank the whole
    search space with the model, time the top 3) is judged on each key's own
    exhaustive sweep (per-configuration median of 5 sweeps, so that the
    exhaustive best is not the luckiest of ~100 single samples).  Asserted:
    its pick reaches >= 0.95 of the exhaustive best (geometric mean), it beats
    the configuration the library runs without tuning (TUNE_DEFAULT), and it
    tunes >= 10x faster than the exhaustive sweep (wall time of
    chai_cuda_tune against the sweep)."""
    dev = ch.Device(config="TopK=3")
    try:
        ctx = dev.ctx
        keys = T.shapes(1040, seed=29, lo=64, hi=2048)
        train, held_keys = keys[:1000], keys[1000:]
        data, _ = T.collect(ctx, train)
        samples = [(k, c) for k, cs in data for c in cs if c.measured_us < 1e29]
        T.train(ctx, samples, epochs=2500, lr=1e-3, seed=1)
        # held-out keys judged on the per-configuration median of 5 sweeps
        held, _ = T.collect(ctx, held_keys, repeats=5)
        rows = T.evaluate(ctx, held)
    finally:
        dev.close()
    gm = lambda v: float(np.exp(np.mean(np.log(np.asarray(v)))))
    pick = gm([r["best_us"] / r["pick_us"] for r in rows])
    dflt = gm([r["best_us"] / r["default_us"] for r in rows])
    speedup = sum(r["exhaustive_s"] for r in rows) / sum(r["learned_s"] for r in rows)
    print("learned pick %.4f of exhaustive best, defaults %.4f, cold start %.1fx" % (pick, dflt, speedup))
    assert pick >= 0.95, (pick, dflt, speedup)
    assert pick > dflt, (pick, dflt)
    assert speedup >= 10.0, speedup


def test_default_mode_reports_the_untuned_configuration(chai_dev):
    """TUNE_DEFAULT: what an untuned call runs, untimed -- CTA-pair 256 x 256
    tiles for large products, one-CTA 128-row tiles for products whose pair
    tiles would leave most SMs idle, the bulk kernel for GEMV."""
    ctx = chai_dev.ctx
    big = T.tune(ctx, T.key(16384, 16384, 16384, L.GEMM_BF16X3), L.TUNE_DEFAULT)
    assert T.cfg_id(big) == (256, 256, 128, 4, 4, 16) and big.cluster_m == 2 and big.measured_us == 0
    small = T.tune(ctx, T.key(512, 512, 512, L.GEMM_BF16X3), L.TUNE_DEFAULT)
    assert (small.block_m, small.block_n, small.cluster_m) == (128, 64, 1)
    # 4 x 16 pair tiles keep 128 SMs busy: pair tiles
    mid = T.tune(ctx, T.key(1024, 4096, 512, L.GEMM_BF16), L.TUNE_DEFAULT)
    assert (mid.block_m, mid.block_n) == (256, 256)
    gv = T.tune(ctx, T.key(4096, 4096, is_gemv=True, precision=L.GEMM_FP32), L.TUNE_DEFAULT)
    assert T.cfg_id(gv) == (0, 0, 0, 0, 1, 0)
    # the small default is a point of the search space
    k = T.key(512, 512, 512, L.GEMM_BF16X3)
    assert T.cfg_id(small) in {T.cfg_id(x) for x in T.sweep(ctx, k)}
