"""Benchmark of the chai B200 back end (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workloads (synthetic, seeded; shapes from the reference's benchmark configs):
  gemm    square f32 GEMM through the trace path's GEMM entry point
          (chai_cuda_gemm), M = N = K = 8192 by default, split-precision bf16x3
          on tcgen05 (--precision to change), the GEMM/GEMV precision sweep case
  mc      Monte Carlo trace: 2^27 Philox4x32-10 Box-Muller normals,
          S = 100 exp(0.03 + 0.2 Z), payoff = mean(max(S - 100, 0)), fully
          fused into one kernel + FP64 combine
  kirsch  8-direction Kirsch compass filter through gather2_floor over an
          8192 x 8192 f32 image (HBM-bound element trace)
  gemv    y = A x, 8192 x 8192 f32 (HBM-bound)

`value` is device-resident throughput (inputs already in HBM, CUDA events on
the context stream, max over ranks); `e2e` is the same metric through the
public API with host buffers, host<->device copies inside the timed region.
`--impl reference` times the reference's own CPU interpreter (built from the
reference sources into oracle/_ref) on a bounded sample of the same workload.
With N > 1 ranks (torchrun) each rank runs the same per-GPU workload on its
own GPU with no collective on the data path ("weak" scaling: traces are
independent), timed between barriers.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers

def lib_and_ctx(config=None):
    from chai_b200 import _lib as L
    ctx = C.c_void_p()
    L.check(L.lib().chai_cuda_init(0, config.encode() if config else None, C.byref(ctx)))
    return L, ctx


def time_events(fn, steps, stream, flush=None):
    """Per-step device time with CUDA events on the launching stream."""
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        if flush is not None:
            flush()
        evs[i][0].record(stream)
        fn()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def l2_flusher():
    import torch
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        buf.zero_()
    return flush


# ---------------------------------------------------------------- workloads

def run_gemm(args, L, ctx, stream):
    import torch
    n = args.size or 8192
    prec = {"fp32": 0, "tf32": 1, "bf16": 2, "bf16x3": 3, "bf16x6": 4, "fp8": 5}[args.precision]
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.rand((n, n), device="cuda", generator=g, dtype=torch.float32) * 2 - 1
    B = torch.rand((n, n), device="cuda", generator=g, dtype=torch.float32) * 2 - 1
    Cm = torch.empty((n, n), device="cuda", dtype=torch.float32)
    d = L.chai_gemm_desc(prec, 0, 0, 0, n, n, n, A.data_ptr(), n, B.data_ptr(), n, Cm.data_ptr(), n, 1.0, 0.0, 1,
                         0, 0, 0)

    def step():
        L.check(L.lib().chai_cuda_gemm(ctx, C.byref(d)), ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    flops = 2.0 * n ** 3
    with Clocks(torch.cuda.current_device()) as clk:
        ts = time_events(step, args.steps, stream)
    ms = sum(ts) / len(ts)
    # e2e: host buffers in, result out, through the public entry point
    Ah, Bh = A.cpu().numpy(), B.cpu().numpy()
    Ch = np.empty((n, n), dtype=np.float32)
    ids = (901, 902, 903)
    for i, arr in zip(ids, (Ah, Bh)):
        L.check(L.lib().chai_cuda_buffer_alloc(ctx, i, arr.nbytes), ctx)
    L.check(L.lib().chai_cuda_buffer_alloc(ctx, ids[2], Ch.nbytes), ctx)
    ptrs = []
    for i in ids:
        p = C.c_void_p()
        L.lib().chai_cuda_buffer_info(ctx, i, C.byref(p), None)
        ptrs.append(p.value)
    de = L.chai_gemm_desc(prec, 0, 0, 0, n, n, n, ptrs[0], n, ptrs[1], n, ptrs[2], n, 1.0, 0.0, 1, 0, 0, 0)

    def e2e():
        L.check(L.lib().chai_cuda_upload(ctx, ids[0], Ah.ctypes.data_as(C.c_void_p), Ah.nbytes), ctx)
        L.check(L.lib().chai_cuda_upload(ctx, ids[1], Bh.ctypes.data_as(C.c_void_p), Bh.nbytes), ctx)
        L.check(L.lib().chai_cuda_gemm(ctx, C.byref(de)), ctx)
        L.check(L.lib().chai_cuda_readback(ctx, ids[2], Ch.ctypes.data_as(C.c_void_p), Ch.nbytes), ctx)

    e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    esteps = max(1, min(args.steps, 5))
    for _ in range(esteps):
        e2e()
    torch.cuda.synchronize()
    e_ms = (time.perf_counter() - t0) * 1e3 / esteps
    P, kind = peaks()
    tensor_mult = {0: 0, 1: 1, 2: 1, 3: 3, 4: 6, 5: 1}[prec]
    achieved = flops * max(1, tensor_mult) / (ms * 1e-3) / 1e12
    return {
        "metric": "GEMM TFLOP/s at err vs FP32", "unit": "TFLOP/s", "value": flops / (ms * 1e-3) / 1e12,
        "ms_per_step": ms, "dtype": args.precision, "higher_is_better": True,
        "config": {"workload": "gemm M=N=K=%d f32 in, %s" % (n, args.precision), "m": n, "n": n, "k": n,
                   "l2": "inputs (%d MiB each) larger than L2" % (n * n * 4 >> 20)},
        "e2e": {"value": flops / (e_ms * 1e-3) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 2 * n * n * 4,
                "d2h_bytes_per_step": n * n * 4},
        "roofline": {"bound": "tensor" if prec else "fp32-simt", "achieved": achieved,
                     "peak": P["bf16_tflops"] if prec else None, "unit": "TFLOP/s",
                     "frac": (achieved / P["bf16_tflops"]) if prec else None, "traffic": None,
                     "peak_source": kind},
        "clocks": clk.summary(), "gpu_launches": args.steps * (2 if prec in (3, 4, 5) else 1),
    }


def mc_expr(ch, g, W, H):
    f = np.float32
    return ch.mean(ch.max(f(100) * ch.exp(f(0.05 - 0.5 * 0.2 * 0.2) + f(0.2) * ch.rng_normal_make(g, W, H))
                          - f(100), f(0)))


def run_mc(args, L, ctx, stream):
    import torch
    import chai_b200.api as ch
    W, H = 8192, 16384                 # 2^27 normals from 2^26 Box-Muller pairs
    dev = ch.init()
    n = W * H
    g = ch.RNGf32(ch.RNG_PHILOX, 42)
    # record the trace once (as the scheduler does for a repeated hash)
    ch._Client.pending = []
    p = ch.Arrayf32(mc_expr(ch, g, W, H))
    stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    ch._Client.pending = []
    bid = 77001
    binds = [(p.var, L.F32 if hasattr(L, "F32") else 4, 1, 1, 1, 0, bid)]
    desc, keep = ch.build_desc(stmts)
    barr = (L.chai_buffer_binding * 1)(L.chai_buffer_binding(*binds[0]))

    def step():
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr, 1), dev.ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        ts = time_events(step, args.steps, stream)
    ms = sum(ts) / len(ts)
    out = np.zeros(1, dtype=np.float32)
    L.check(L.lib().chai_cuda_readback(dev.ctx, bid, out.ctypes.data_as(C.c_void_p), 4), dev.ctx)

    # e2e through the public API: record + evaluate + read_scalar each step
    def e2e():
        g2 = ch.RNGf32(ch.RNG_PHILOX, 42)
        return float(ch.Arrayf32(mc_expr(ch, g2, W, H)).read_scalar())

    e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    esteps = max(1, args.steps)
    for _ in range(esteps):
        payoff = e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / esteps
    return {
        "metric": "trace throughput (MC: Philox normals -> exp -> mean)", "unit": "Gnormals/s",
        "value": n / (ms * 1e-3) / 1e9, "ms_per_step": ms, "dtype": "f32", "higher_is_better": True,
        "config": {"workload": "mc 2^27 normals fused", "normals": n, "payoff": payoff,
                   "l2": "no HBM inputs (RNG in registers)"},
        "e2e": {"value": n / (e_ms * 1e-3) / 1e9, "unit": "Gnormals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 16},
        "roofline": None, "clocks": clk.summary(), "gpu_launches": args.steps * 2,
    }


WORKLOADS = {"gemm": run_gemm, "mc": run_mc}


# ---------------------------------------------------------------- reference arm

def run_reference(args):
    """The reference's own CPU interpreter (oracle/_ref/ref_driver), on a
    bounded sample of the same workload."""
    drv = ROOT / "oracle" / "_ref" / "ref_driver"
    cores = 1   # the interpreter device is one thread (runtime/DeviceMap.cpp:17-23)
    if not drv.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_driver not built"}
    wl = args.workload
    with tempfile.TemporaryDirectory() as td:
        if wl == "gemm":
            n = 1024
            rng = np.random.default_rng(1)
            A = rng.uniform(-1, 1, (n, n)).astype(np.float32)
            A.tofile(td + "/A")
            A.tofile(td + "/B")
            times = []
            for _ in range(max(1, min(args.steps, 3))):
                r = subprocess.run([str(drv), "gemm_f32", str(n), str(n), str(n), td + "/A", td + "/B", td + "/C"],
                                   capture_output=True, text=True, timeout=600)
                times.append(float(r.stdout.split("ms=")[1].split()[0]))
            ms = statistics.median(times)
            v = 2.0 * n ** 3 / (ms * 1e-3) / 1e12
            unit, metric = "TFLOP/s", "GEMM TFLOP/s at err vs FP32"
            sample = "interpreter matmul 1024^3 f32 (double accumulation), make2 inputs"
        else:
            W, H = 1024, 1024
            times = []
            for _ in range(max(1, min(args.steps, 3))):
                r = subprocess.run([str(drv), "mc_rng", str(W), str(H)], capture_output=True, text=True,
                                   timeout=600)
                times.append(float(r.stdout.split("ms=")[1].split()[0]))
            ms = statistics.median(times)
            v = W * H / (ms * 1e-3) / 1e9
            unit, metric = "Gnormals/s", "trace throughput (MC: Philox normals -> exp -> mean)"
            sample = "interpreter MC trace over 2^20 normals (its own RNG)"
    return {"impl": "reference", "metric": metric, "value": v, "unit": unit, "ms_per_step": ms,
            "higher_is_better": True, "cpu_baseline": {"value": v, "unit": unit, "cores": cores,
                                                      "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline(args):
    r = run_reference(args)
    return r.get("cpu_baseline") if "cpu_baseline" in r else None


# ---------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="gemm", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--size", type=int, default=0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            line = run_reference(args)
            line.update({"n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup})
            print(json.dumps(line))
        return
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    from chai_b200 import _lib as L
    import chai_b200.api as ch
    dev = ch.init(device=local)
    stream = torch.cuda.Stream()          # one stream shared by torch events and the library
    torch.cuda.set_stream(stream)
    L.lib().chai_cuda_set_stream(dev.ctx, C.c_void_p(stream.cuda_stream))
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    res = WORKLOADS[args.workload](args, L, dev.ctx, stream)
    torch.cuda.synchronize()
    ms = res["ms_per_step"]
    if pg:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        res["value"] = res["value"] * world * res["ms_per_step"] / ms
        res["ms_per_step"] = ms
    if rank == 0:
        line = {"metric": res["metric"], "value": res["value"], "unit": res["unit"], "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": res["higher_is_better"], "scaling": "weak", "vs_baseline": None,
                "dtype": res["dtype"], "data": "synthetic (seeded)",
                "config": dict(res["config"], parallelism="independent traces per GPU (dp%d)" % world)}
        for k in ("e2e", "roofline", "clocks", "gpu_launches"):
            line[k] = res.get(k)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    ch.shutdown()


if __name__ == "__main__":
    main()
