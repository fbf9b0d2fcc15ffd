"""Sharding helpers (chai_b200/shard.py) as gloo ranks on CPU, world sizes 2
and 3, one process per rank as torch.distributed.run starts them on GPUs.
The per-rank compute is the oracle (test side only); the exchanges are the
product's: halo rows for a row-sharded Kirsch stencil, B broadcast for a
row-sharded GEMM, one all-reduce for a sharded sum, the partitioned tuning
sweep."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

from chai_b200 import shard  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _image(H, W, seed=5):
    return np.random.default_rng(seed).random((H, W), dtype=np.float32)


def _rank(rank, world, port, H, W, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from chai_b200 import _lib as L
    from chai_b200 import shard as S
    from oracle import cpu as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {}
        img = _image(H, W)
        # Kirsch on a row shard with a one-row halo from the neighbours
        r0, r1 = S.split(H, world, rank)
        slab = S.stencil_slab(torch.from_numpy(img[r0:r1].copy()), 1)
        res["slab"] = slab.numpy()
        res["kirsch"] = S.crop(torch.from_numpy(O.kirsch(slab.numpy())), 1).numpy()
        res["kirsch_all"] = S.gather_rows(torch.from_numpy(res["kirsch"]), H).numpy()
        # row-sharded GEMM: rank 0 holds B; C rows gathered in rank order
        rng = np.random.default_rng(9)
        M, K, N = 37, 24, 19
        A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
        B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
        a0, a1 = S.split(M, world, rank)
        c_rows = S.gemm_rows(torch.from_numpy(A[a0:a1].copy()), torch.from_numpy(B) if rank == 0 else None, N,
                             compute=lambda a, b: torch.from_numpy(O.matmul_ref(a.numpy(), b.numpy())))
        res["gemm"] = S.gather_rows(c_rows, M).numpy()
        # sharded FP64 sum
        x = rng.uniform(0, 1, 1001)
        x0, x1 = S.split(len(x), world, rank)
        res["sum"] = S.sum_shards(float(np.sum(x[x0:x1], dtype=np.float64)))
        # partitioned tuning sweep with a stand-in timing function
        keys = [L.chai_gemm_key(64 * (i + 1), 128, 32 * (i % 3 + 1), L.GEMM_BF16X3, 0) for i in range(7)]
        calls = []

        def sweep(k):
            calls.append(int(k.m))
            return [L.chai_gemm_cfg(128, bn, 64, 4, 1, 1, 1, 16, float(k.m * bn) / 1000) for bn in (128, 256)]
        merged = S.sweep_sharded(keys, sweep)
        res["sweep"] = [(int(k.m), [(c.block_n, c.measured_us) for c in cs]) for k, cs in merged]
        res["sweep_calls"] = calls
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world, H=13, W=16):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, H, W, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    return {r: out[r] for r in range(world)}


def test_split_is_contiguous_and_balanced():
    for n in (0, 1, 7, 13, 1000):
        for world in (1, 2, 3, 8):
            parts = [shard.split(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.split(5, 2, 2)


def test_single_rank_slab_wraps_periodically():
    img = torch.arange(12, dtype=torch.float32).reshape(4, 3)
    slab = shard.stencil_slab(img, 1)
    assert torch.equal(slab[0], img[3]) and torch.equal(slab[-1], img[0]) and torch.equal(slab[1:5], img)
    with pytest.raises(ValueError):
        shard.stencil_slab(img[:1], 2)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_stencil_gemm_sum_and_sweep_match_one_rank(world):
    from oracle import cpu as O
    H, W = 13, 16
    res = _run(world, H, W)
    img = _image(H, W)
    full = O.kirsch(img)
    for r in range(world):
        r0, r1 = shard.split(H, world, r)
        rows = [(y % H) for y in range(r0 - 1, r1 + 1)]
        assert np.array_equal(res[r]["slab"], img[rows])          # halo rows from both neighbours
        assert np.array_equal(res[r]["kirsch"], full[r0:r1])      # bit-exact against the whole image
        assert np.array_equal(res[r]["kirsch_all"], full)
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (37, 24)).astype(np.float32)
    B = rng.uniform(-1, 1, (24, 19)).astype(np.float32)
    x = rng.uniform(0, 1, 1001)
    ref = O.matmul_ref(A, B)
    for r in range(world):
        assert np.array_equal(res[r]["gemm"], ref)
        assert res[r]["sum"] == pytest.approx(float(np.sum(x)), rel=1e-14)
        assert res[r]["sweep_calls"] == [64 * (i + 1) for i in range(r, 7, world)]
        assert res[r]["sweep"] == [(64 * (i + 1), [(bn, 64 * (i + 1) * bn / 1000) for bn in (128, 256)])
                                   for i in range(7)]
