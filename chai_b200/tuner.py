"""Offline / cold-start GEMM and GEMV tuning through the C ABI.

The host side of the tuner: the exhaustive sweep that generates the cost
model's training data (the role of tools/ATmatmul.cpp and tools/ATmatvec.cpp,
which drive StandardEM::searchLoop, autotune/StandardEM.cpp:69-121), training
of the MLP cost model on the GPU, and learned (top-k) versus exhaustive tuning
of new shapes.  Every timing and every network pass runs in the CUDA library
(chai_b200/csrc/tuner.cpp, chai_b200/csrc/mlp.cu).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib as L

N_FEATURES = 14
GEMM_SPACE = 104
GEMV_SPACE = 17


def key(m, n, k=1, precision=L.GEMM_BF16X3, is_gemv=False) -> L.chai_gemm_key:
    return L.chai_gemm_key(int(m), int(n), 1 if is_gemv else int(k),
                           L.GEMM_FP64 if (is_gemv and precision == L.GEMM_FP64) else int(precision),
                           1 if is_gemv else 0)


def shapes(count: int, seed: int = 13, lo: int = 64, hi: int = 16384, gemv_frac: float = 0.25,
           precisions=(L.GEMM_FP32, L.GEMM_BF16)):
    """`count` tuning keys with M, N, K log-uniform in [lo, hi] (rounded to
    multiples of 8), dtype alternating over `precisions`; a fraction are GEMV
    (f32) keys."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m, n, k = (int(max(lo, min(hi, round(math.exp(rng.uniform(math.log(lo), math.log(hi))) / 8) * 8)))
                   for _ in range(3))
        if rng.uniform() < gemv_frac:
            out.append(key(m, n, is_gemv=True, precision=L.GEMM_FP32))
        else:
            out.append(key(m, n, k, precision=precisions[i % len(precisions)]))
    return out


def sweep(ctx, k: L.chai_gemm_key):
    """Time every configuration of the search space for `k` (list of cfgs)."""
    buf = (L.chai_gemm_cfg * 256)()
    n = C.c_int(0)
    L.check(L.lib().chai_cuda_tune_sweep(ctx, C.byref(k), buf, 256, C.byref(n)), ctx)
    return [L.chai_gemm_cfg.from_buffer_copy(buf[i]) for i in range(n.value)]


def tune(ctx, k: L.chai_gemm_key, mode=L.TUNE_LEARNED) -> L.chai_gemm_cfg:
    out = L.chai_gemm_cfg()
    L.check(L.lib().chai_cuda_tune(ctx, C.byref(k), int(mode), C.byref(out)), ctx)
    return out


def features(k: L.chai_gemm_key, cfg: L.chai_gemm_cfg) -> np.ndarray:
    f = (C.c_float * N_FEATURES)()
    L.check(L.lib().chai_cuda_tune_features(C.byref(k), C.byref(cfg), f))
    return np.frombuffer(f, dtype=np.float32).copy()


def _arrays(samples):
    keys = (L.chai_gemm_key * len(samples))(*[s[0] for s in samples])
    cfgs = (L.chai_gemm_cfg * len(samples))(*[s[1] for s in samples])
    return keys, cfgs


def train(ctx, samples, epochs=3000, lr=1e-3, seed=1) -> float:
    """Train the cost model on [(key, cfg with measured_us)]; returns the
    final training loss (MSE on standardised log runtime)."""
    keys, cfgs = _arrays(samples)
    loss = C.c_double(0)
    L.check(L.lib().chai_cuda_mlp_train(ctx, keys, cfgs, len(samples), int(epochs), float(lr), int(seed),
                                        C.byref(loss)), ctx)
    return loss.value


def predict(ctx, samples) -> np.ndarray:
    """Predicted log(us) for [(key, cfg)]."""
    keys, cfgs = _arrays(samples)
    out = (C.c_double * len(samples))()
    L.check(L.lib().chai_cuda_mlp_predict(ctx, keys, cfgs, len(samples), out), ctx)
    return np.frombuffer(out, dtype=np.float64).copy()


def gradients(ctx, samples):
    keys, cfgs = _arrays(samples)
    n = weight_count(ctx) - 2
    g = (C.c_float * n)()
    loss = C.c_double(0)
    L.check(L.lib().chai_cuda_mlp_gradients(ctx, keys, cfgs, len(samples), g, n, C.byref(loss)), ctx)
    return loss.value, np.frombuffer(g, dtype=np.float32).copy()


def weight_count(ctx) -> int:
    c = C.c_size_t(0)
    L.check(L.lib().chai_cuda_mlp_weights(ctx, None, 0, C.byref(c), 0), ctx)
    return c.value


def get_weights(ctx) -> np.ndarray:
    n = weight_count(ctx)
    buf = (C.c_float * n)()
    c = C.c_size_t(0)
    L.check(L.lib().chai_cuda_mlp_weights(ctx, buf, n, C.byref(c), 0), ctx)
    return np.frombuffer(buf, dtype=np.float32).copy()


def set_weights(ctx, w: np.ndarray):
    w = np.ascontiguousarray(w, dtype=np.float32)
    c = C.c_size_t(0)
    L.check(L.lib().chai_cuda_mlp_weights(ctx, w.ctypes.data_as(C.POINTER(C.c_float)), w.size, C.byref(c), 1), ctx)


def sweep_median(ctx, k: L.chai_gemm_key, repeats: int):
    """`repeats` sweeps of `k`; each configuration's time is its median.  The
    best of a single sweep is the minimum of ~100 noisy samples and reads
    optimistic; judging picks against medians removes that bias."""
    runs = [sweep(ctx, k) for _ in range(repeats)]
    out = runs[0]
    by = {}
    for r in runs:
        for c in r:
            by.setdefault(cfg_id(c), []).append(c.measured_us)
    for c in out:
        c.measured_us = float(np.median(by[cfg_id(c)]))
    return out


def collect(ctx, keys, log=None, repeats=1):
    """Exhaustive sweep over `keys` (per-configuration median of `repeats`
    sweeps): returns [(key, [cfg...])] and seconds."""
    t0 = time.perf_counter()
    out = []
    for i, k in enumerate(keys):
        out.append((k, sweep(ctx, k) if repeats <= 1 else sweep_median(ctx, k, repeats)))
        if log and (i + 1) % 100 == 0:
            log("swept %d/%d keys (%.1f s)" % (i + 1, len(keys), time.perf_counter() - t0))
    return out, time.perf_counter() - t0


def cfg_id(c: L.chai_gemm_cfg):
    return (c.block_m, c.block_n, c.block_k, c.stages, c.vec_width, c.group_m)


def evaluate(ctx, held_out, default_ids=None):
    """Learned top-k tuning of held-out keys judged against their exhaustive
    sweeps: per key, the best time over the sweep, the sweep's own time for the
    learned pick and for the default configuration (what an untuned call of
    that shape runs, TUNE_DEFAULT), and the wall time of each method (learned:
    ranking + timing the top k; exhaustive: the sweep)."""
    rows = []
    # size every operand / scratch buffer for the largest key first, so that
    # neither method's timing includes a first-touch allocation
    for gemv in (0, 1):
        ks = [k for k, _ in held_out if k.is_gemv == gemv]
        for prec in sorted({k.precision for k in ks}):
            sub = [k for k in ks if k.precision == prec]
            sweep(ctx, key(max(k.m for k in sub), max(k.n for k in sub), max(k.k for k in sub), prec, bool(gemv)))
    for k, cfgs in held_out:
        by_id = {cfg_id(c): c.measured_us for c in cfgs}
        best = min(by_id.values())
        t0 = time.perf_counter()
        pick = tune(ctx, k, L.TUNE_LEARNED)
        t_learned = time.perf_counter() - t0
        t0 = time.perf_counter()
        sweep(ctx, k)
        t_exh = time.perf_counter() - t0
        dflt = cfg_id(tune(ctx, k, L.TUNE_DEFAULT))
        rows.append(dict(m=k.m, n=k.n, k=k.k, precision=k.precision, gemv=k.is_gemv, best_us=best,
                         pick_us=by_id.get(cfg_id(pick), float("nan")),
                         default_us=by_id.get(dflt, float("nan")), learned_s=t_learned, exhaustive_s=t_exh))
    return rows
