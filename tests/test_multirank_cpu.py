"""The multi-rank host logic of bench.py on CPU: world-size-2 gloo ranks
(one process per rank, as torch.distributed.run starts them on GPUs) with
different step times; rank 0's whole-job value must be the units both ranks
processed divided by the slower rank's time (weak scaling, max over ranks)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        units = 1000.0                      # per-rank work per step
        ms = 2.0 + rank                     # rank 1 is slower
        res = {"value": units / ms, "ms_per_step": ms, "e2e": {"value": 10.0 - rank, "unit": "x"}}

        def reduce_max(x):
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        bench.aggregate_ranks(res, world, reduce_max)
        out[rank] = (res["value"], res["ms_per_step"], res["e2e"]["value"])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_weak_scaling_value_is_total_units_over_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        value, ms, e2e = out[r]
        assert ms == pytest.approx(3.0)
        assert value == pytest.approx(2 * 1000.0 / 3.0)
        assert e2e == pytest.approx(2 * 9.0)          # the slowest rank's end-to-end rate, times the ranks
