"""Tuner host logic on the CPU: the library's feature map against the oracle's
restatement, the search space, and the oracle MLP's backward pass against
central finite differences (which pins the oracle used by the GPU gradient
check in test_gpu_tuner.py)."""
import numpy as np
import pytest

from chai_b200 import _lib as L
from chai_b200 import tuner as T
from oracle import mlp as OM


def _cfg(d):
    c = L.chai_gemm_cfg()
    for k, v in d.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("is_gemv", [False, True])
def test_features_match_oracle(is_gemv):
    rng = np.random.default_rng(5)
    for _ in range(60):
        m, n, k = (int(x) for x in rng.integers(1, 20000, 3))
        prec = int(rng.choice([L.GEMM_FP32, L.GEMM_BF16, L.GEMM_BF16X3, L.GEMM_TF32]))
        for d in OM.space(is_gemv):
            key = T.key(m, n, k, prec, is_gemv)
            got = T.features(key, _cfg(d))
            want = OM.features(key.m, key.n, key.k, key.precision, is_gemv, d)
            np.testing.assert_allclose(got, want, rtol=2e-7, atol=0)


def test_search_space_sizes():
    assert len(OM.space(False)) == T.GEMM_SPACE
    assert len(OM.space(True)) == T.GEMV_SPACE
    assert OM.count() == 14 * 128 + 128 + 2 * (128 * 128 + 128) + 128 + 1
    assert T.GEMM_SPACE >= 100


def test_tuning_shapes_are_log_uniform_and_seeded():
    ks = T.shapes(400, seed=13)
    assert [(k.m, k.n, k.k) for k in ks[:5]] == [(k.m, k.n, k.k) for k in T.shapes(5, seed=13)]
    dims = np.array([[k.m, k.n] for k in ks], dtype=np.float64)
    assert dims.min() >= 64 and dims.max() <= 16384
    assert np.all(dims % 8 == 0)
    # log-uniform: the median of log2 sits near the middle of [6, 14]
    assert abs(np.median(np.log2(dims)) - 10.0) < 0.6
    gemv = sum(k.is_gemv for k in ks)
    assert 60 < gemv < 140


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = OM.init(7).astype(np.float64)
    w[-2:] = [0.3, 1.7]                         # mean, scale
    x = rng.uniform(0, 1, (24, OM.IN))
    y = rng.normal(0, 1, 24)
    _, g = OM.loss_and_grads(w, x, y)
    idx = rng.choice(OM.count(), 40, replace=False)
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        num = (OM.loss_and_grads(wp, x, y)[0] - OM.loss_and_grads(wm, x, y)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])
