"""Sharding traced array programs over several GPUs of one node.

One process per GPU; `torch.distributed` carries the exchanges (NCCL between
GPUs, gloo for CPU ranks).  The reference runs all traces of a process on the
devices of one host, one device thread each (`runtime/Scheduler.cpp:102-186`,
`runtime/DeviceMap.cpp:12-36`), and never exchanges data between devices: a
trace (and each slot of a vectorised trace) is independent work.  Whole
traces therefore shard with no exchange at all.  The helpers here cover the
cases where one large object is split across ranks:

- `split(n, world, rank)`: the contiguous, balanced share of `n` units.
- `stencil_slab(own, halo)`: a rank owning rows [r0, r1) of an image gets
  `halo` rows from each neighbour (periodic in rows, as `gather2_floor` wraps,
  `interp/InterpGather.hpp:36-42`) by point-to-point messages.  A
  constant-offset stencil trace evaluated on the slab gives exactly the global
  result on rows [halo, halo + r1 - r0) of the slab (`crop`): its gathers at
  row offsets within +-halo never reach the slab's own wrap.
- `gemm_rows(...)`: C rows [r0, r1) = A rows [r0, r1) times B.  B is
  broadcast once from rank 0 into every rank's own memory before the GEMM,
  so no GEMM kernel ever reads another GPU's memory.
- `sum_shards(partial)`: each rank reduces its shard in FP64; one all-reduce
  of one double combines them.
- `sweep_sharded(keys, sweep)`: the exhaustive tuning sweep partitioned
  round-robin over ranks; results are all-gathered and every rank gets the
  full list in key order.
"""
from __future__ import annotations

import ctypes as C

import torch
import torch.distributed as dist

from . import _lib as L


def _world(group=None):
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def split(n: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of rank `rank`'s contiguous share of `n` units; the
    first n % world ranks take one unit more."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("split: bad n=%d world=%d rank=%d" % (n, world, rank))
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def stencil_slab(own: torch.Tensor, halo: int = 1, group=None) -> torch.Tensor:
    """Rows [r0 - halo, r1 + halo) of a row-sharded image whose rows wrap
    periodically, from this rank's rows `own` ([r1 - r0, W]).

    Ranks are ordered by rank number along the rows: rank r's last rows are
    rank r+1's top halo, its first rows rank r-1's bottom halo (ring).  Each
    rank sends two `halo`-row messages and receives two.  Every rank must own
    at least `halo` rows."""
    if own.dim() != 2:
        raise ValueError("stencil_slab: own rows must be a 2-D [rows, W] tensor")
    h = own.shape[0]
    if halo < 0 or h < halo:
        raise ValueError("stencil_slab: %d rows cannot supply a halo of %d" % (h, halo))
    if halo == 0:
        return own.contiguous()
    world, rank = _world(group)
    if world == 1:
        return torch.cat([own[h - halo:], own, own[:halo]]).contiguous()
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    last = own[h - halo:].contiguous()
    first = own[:halo].contiguous()
    top = torch.empty_like(first)
    bottom = torch.empty_like(first)
    # Per peer pair the messages are posted in the same order on both sides
    # (NCCL matches point-to-point operations by order, not by tag): a rank
    # sends its last rows before its first rows and receives its top halo
    # before its bottom halo.  With two ranks prev == nxt and the order still
    # matches: the peer's last rows arrive first and become the top.
    ops = [dist.P2POp(dist.isend, last, nxt, group, 1),
           dist.P2POp(dist.isend, first, prev, group, 2),
           dist.P2POp(dist.irecv, top, prev, group, 1),
           dist.P2POp(dist.irecv, bottom, nxt, group, 2)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    return torch.cat([top, own, bottom]).contiguous()


def crop(slab_out: torch.Tensor, halo: int = 1) -> torch.Tensor:
    """The rows of a stencil result on a slab that belong to this rank."""
    return slab_out[halo:slab_out.shape[0] - halo] if halo else slab_out


def broadcast_operand(b: torch.Tensor | None, shape, dtype, device, group=None, src: int = 0) -> torch.Tensor:
    """`b` from rank `src` in every rank's own memory (other ranks pass None)."""
    world, rank = _world(group)
    if rank == src:
        if b is None:
            raise ValueError("broadcast_operand: the source rank must supply the operand")
        b = b.contiguous()
        if world > 1:
            dist.broadcast(b, src, group)
        return b
    out = torch.empty(shape, dtype=dtype, device=device)
    dist.broadcast(out, src, group)
    return out


def _chai_gemm(ctx, precision: int):
    def run(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        if a.device.type != "cuda" or b.device.type != "cuda":
            raise RuntimeError("gemm_rows: operands must be CUDA tensors for the chai_b200 GEMM")
        m, k = a.shape
        n = b.shape[1]
        c = torch.empty((m, n), dtype=torch.float32, device=a.device)
        if m:
            d = L.chai_gemm_desc(precision, 0, 0, 0, m, n, k, a.data_ptr(), k, b.data_ptr(), n, c.data_ptr(), n,
                                 1.0, 0.0, 1, 0, 0, 0)
            L.check(L.lib().chai_cuda_gemm(ctx, C.byref(d)), ctx)
        return c
    return run


def gemm_rows(a_rows: torch.Tensor, b: torch.Tensor | None, n: int, *, ctx=None, precision: int = L.GEMM_AUTO,
              compute=None, group=None) -> torch.Tensor:
    """This rank's rows of C = A B (f32, row-major).

    `a_rows` holds this rank's rows of A ([m_r, K]); rank 0 passes B ([K, n]),
    the other ranks None.  B is broadcast into local memory first, then the
    local GEMM runs on local operands only.  `compute(a, b)` defaults to
    `chai_cuda_gemm` on `ctx`."""
    k = a_rows.shape[1]
    b = broadcast_operand(b, (k, n), torch.float32, a_rows.device, group)
    if compute is None:
        if ctx is None:
            raise ValueError("gemm_rows: pass ctx (a chai_b200 context) or compute")
        compute = _chai_gemm(ctx, precision)
    return compute(a_rows.contiguous(), b)


def gather_rows(part: torch.Tensor, total_rows: int, group=None) -> torch.Tensor:
    """All ranks' row blocks (split by `split`) concatenated in rank order."""
    world, rank = _world(group)
    if world == 1:
        return part
    rows = max(split(total_rows, world, r)[1] - split(total_rows, world, r)[0] for r in range(world))
    pad = torch.zeros((rows,) + tuple(part.shape[1:]), dtype=part.dtype, device=part.device)
    pad[:part.shape[0]] = part
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group)
    out = []
    for r in range(world):
        s, e = split(total_rows, world, r)
        out.append(bufs[r][:e - s])
    return torch.cat(out)


def sum_shards(partial: float, group=None, device=None) -> float:
    """Sum of every rank's FP64 partial (one all-reduce of one double)."""
    world, _ = _world(group)
    if world == 1:
        return float(partial)
    t = torch.tensor([float(partial)], dtype=torch.float64, device=device)
    dist.all_reduce(t, dist.ReduceOp.SUM, group)
    return float(t.item())


def sweep_sharded(keys, sweep, group=None):
    """Exhaustive tuning sweep over `keys`, keys i with i % world == rank on
    this rank; returns [(key, [cfg...])] in key order on every rank.

    `sweep(key)` times every configuration of one key (for example
    `chai_b200.tuner.sweep` bound to a context).  Keys and configurations are
    ctypes structures; they cross ranks as their raw bytes."""
    world, rank = _world(group)
    mine = []
    for i in range(rank, len(keys), world):
        mine.append((i, [bytes(c) for c in sweep(keys[i])]))
    if world == 1:
        got = [mine]
    else:
        got = [None] * world
        dist.all_gather_object(got, mine, group)
    by_index = {}
    for part in got:
        for i, cfgs in part:
            by_index[i] = [L.chai_gemm_cfg.from_buffer_copy(c) for c in cfgs]
    if sorted(by_index) != list(range(len(keys))):
        raise RuntimeError("sweep_sharded: missing results for some keys")
    return [(keys[i], by_index[i]) for i in range(len(keys))]
