"""CPU restatement (numpy, float64) of the tuner's cost model: the feature map,
the search space, and the MLP forward pass, loss and backward pass.

Test infrastructure only: the parity tests check the library's GPU forward /
backward kernels (chai_b200/csrc/mlp.cu) and its feature map
(chai_b200/csrc/tuner.cpp) against these functions.

The reference has no learned model: its tuner times every candidate of an
alternating coordinate search (autotune/StandardEM.cpp:69-147,
autotune/AutoTuneBench.cpp:17-251).  What this file restates is therefore this
library's own definition of the model, which the tuner uses to rank the
candidates of that search before timing the top k:

  features (14): log2 M/14, log2 N/14, log2 K/14 (K = 1 for GEMV), split
    precision (fp32 via bf16x3) flag, single-pass tensor-core flag, GEMV flag,
    CTA-pair flag (block_m 256), block_n/256, stages/8, log2(group_m)/7, GEMV
    warps/16, GEMV unroll/8, wave efficiency (fraction of the last wave of
    work units with work), tile fill (fraction of the tiles' area inside M x N)
  network: 14 -> 128 -> 128 -> 128 -> 1, ReLU on the hidden layers,
    y = x W + b with W stored row-major (in x out)
  target: (log(measured_us) - mean) / scale, loss = mean squared error
  parameter order: W1 b1 W2 b2 W3 b3 W4 b4, then mean and scale
"""
from __future__ import annotations

import numpy as np

IN, H = 14, 128
DIMS = [IN, H, H, H, 1]
GEMM_FP32, GEMM_TF32, GEMM_BF16, GEMM_BF16X3, GEMM_BF16X6, GEMM_FP8, GEMM_FP64 = range(7)


TILES = [(128, 64, 4), (128, 64, 6), (128, 64, 8), (128, 128, 4), (128, 128, 6), (128, 256, 3), (128, 256, 4),
         (256, 128, 4), (256, 128, 6), (256, 128, 8), (256, 256, 3), (256, 256, 4), (256, 256, 6)]


def space(is_gemv: bool):
    """Search space as dicts of chai_gemm_cfg fields (tuner.cpp Tuner::space)."""
    if is_gemv:
        return [dict(block_m=0, vec_width=1)] + [dict(block_m=w, vec_width=u) for w in (2, 4, 8, 16)
                                                 for u in (1, 2, 4, 8)]
    return [dict(block_m=bm, block_n=bn, block_k=128, stages=st, vec_width=4, group_m=g,
                 cluster_m=2 if bm == 256 else 1, cluster_n=1)
            for bm, bn, st in TILES for g in (1, 2, 4, 8, 16, 32, 64, 128)]


def features(m, n, k, precision, is_gemv, cfg) -> np.ndarray:
    """float32[14] feature vector of (key, cfg)."""
    m, n = max(1, m), max(1, n)
    k = 1 if is_gemv else max(1, k)
    split = precision in (GEMM_BF16X3, GEMM_BF16X6, GEMM_FP32)
    f = np.zeros(IN, dtype=np.float64)
    f[0] = np.log2(m) / 14.0
    f[1] = np.log2(n) / 14.0
    f[2] = np.log2(k) / 14.0
    f[3] = 1.0 if (not is_gemv and split) else 0.0
    f[4] = 1.0 if (not is_gemv and not split) else 0.0
    f[5] = 1.0 if is_gemv else 0.0
    f[6] = 1.0 if (not is_gemv and cfg.get("block_m", 0) == 256) else 0.0
    f[7] = cfg.get("block_n", 0) / 256.0
    f[8] = cfg.get("stages", 0) / 8.0
    g = cfg.get("group_m", 0)
    f[9] = np.log2(g) / 7.0 if g > 0 else 0.0
    f[10] = cfg.get("block_m", 0) / 16.0 if is_gemv else 0.0
    f[11] = cfg.get("vec_width", 0) / 8.0 if is_gemv else 0.0
    f[12] = wave_efficiency(m, n, is_gemv, cfg)
    f[13] = tile_fill(m, n, is_gemv, cfg)
    return f.astype(np.float32)


def wave_efficiency(m, n, is_gemv, cfg) -> float:
    """Fraction of the last wave with work: GEMM tiles of block_m x block_n over
    148 persistent CTAs (74 CTA pairs for block_m 256); GEMV blocks of `warps`
    rows, 64 / warps blocks per SM."""
    if is_gemv:
        w = max(1, cfg.get("block_m", 0))
        units = np.ceil(max(1, m) / w)
        per_wave = 148.0 * max(1, min(32, 64 // w))
    else:
        bm = 256 if cfg.get("block_m", 0) == 256 else 128
        units = np.ceil(max(1, m) / bm) * np.ceil(max(1, n) / max(1, cfg.get("block_n", 0)))
        per_wave = 74.0 if bm == 256 else 148.0
    return units / (np.ceil(units / per_wave) * per_wave)


def tile_fill(m, n, is_gemv, cfg) -> float:
    """Fraction of the tiles' area inside the M x N product."""
    if is_gemv:
        return 0.0
    bm = 256.0 if cfg.get("block_m", 0) == 256 else 128.0
    bn = float(max(1, cfg.get("block_n", 0)))
    return (m * n) / (np.ceil(m / bm) * bm * np.ceil(n / bn) * bn)


def count() -> int:
    return sum(DIMS[i] * DIMS[i + 1] + DIMS[i + 1] for i in range(4))


def unpack(flat):
    """Split a flat parameter vector (+ mean, scale) into [(W, b)], mean, scale."""
    flat = np.asarray(flat, dtype=np.float64)
    layers, off = [], 0
    for i in range(4):
        w = flat[off:off + DIMS[i] * DIMS[i + 1]].reshape(DIMS[i], DIMS[i + 1])
        off += DIMS[i] * DIMS[i + 1]
        b = flat[off:off + DIMS[i + 1]]
        off += DIMS[i + 1]
        layers.append((w, b))
    mean, scale = (flat[off], flat[off + 1]) if flat.size >= off + 2 else (0.0, 1.0)
    return layers, mean, scale


def init(seed: int, rng=None) -> np.ndarray:
    """He-uniform weights, zero biases, mean 0, scale 1 (any seeded init works
    for the parity checks; the library's own init uses its host generator)."""
    rng = rng or np.random.default_rng(seed)
    parts = []
    for i in range(4):
        lim = np.sqrt(6.0 / DIMS[i])
        parts.append(rng.uniform(-lim, lim, DIMS[i] * DIMS[i + 1]))
        parts.append(np.zeros(DIMS[i + 1]))
    parts.append(np.array([0.0, 1.0]))
    return np.concatenate(parts).astype(np.float32)


def forward(flat, x):
    """Standardised prediction (n,) and the activations."""
    layers, _, _ = unpack(flat)
    acts = [np.asarray(x, dtype=np.float64)]
    for i, (w, b) in enumerate(layers):
        z = acts[-1] @ w + b
        acts.append(np.maximum(z, 0.0) if i < 3 else z)
    return acts[-1][:, 0], acts


def predict_log_us(flat, x):
    _, mean, scale = unpack(flat)
    p, _ = forward(flat, x)
    return p * scale + mean


def loss_and_grads(flat, x, log_us):
    """MSE loss on standardised targets and the gradient of every weight, in
    the flat parameter order (without mean and scale)."""
    layers, mean, scale = unpack(flat)
    y = (np.asarray(log_us, dtype=np.float64) - mean) / scale
    p, acts = forward(flat, x)
    n = y.size
    diff = p - y
    loss = float(np.mean(diff * diff))
    d = (2.0 * diff / n)[:, None]
    grads = [None] * 4
    for i in range(3, -1, -1):
        if i < 3:
            d = d * (acts[i + 1] > 0.0)
        w, _ = layers[i]
        grads[i] = (acts[i].T @ d, d.sum(axis=0))
        if i > 0:
            d = d @ w.T
    return loss, np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
