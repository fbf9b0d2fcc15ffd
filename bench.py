"""Benchmark of the chai B200 back end (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workloads (synthetic, seeded; shapes from the reference's benchmark configs):
  gemm    square f32 GEMM through the trace path's GEMM entry point
          (chai_cuda_gemm), M = N = K = 16384 by default, split-precision bf16x3
          on tcgen05 (--precision to change), the GEMM/GEMV precision sweep case
  mc      Monte Carlo trace: 2^27 Philox4x32-10 Box-Muller normals,
          S = 100 exp(0.03 + 0.2 Z), payoff = mean(max(S - 100, 0)), fully
          fused into one kernel + FP64 combine
  kirsch  8-direction Kirsch compass filter through gather2_floor over an
          8192 x 8192 f32 image (HBM-bound element trace)
  gemv    y = A x, 8192 x 8192 f32 (HBM-bound)
  mc-hbm  the materialised Monte Carlo payoff over 2^27 normals in HBM
  mc-many 64 Monte Carlo traces of uneven lengths in one persistent launch
  grouped 4096 grouped f32 GEMMs (M, N, K multiples of 8 in [32, 512])
  tuner   learned vs exhaustive GEMM/GEMV tuning on held-out shapes
  c1      512^3 matmul + sum(C*C) as one traced program (latency-bound)

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
import math
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once the sampler is printing (start-up
            # of nvidia-smi takes a good part of a short region otherwise)
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.skip = len(self.lines)
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
        for ln in self.lines[getattr(self, "skip", 0):]:
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


def timed_region(fn, args, stream):
    """The timed region of a workload: `args.steps` steps, or -- when
    `args.min_timed_s` is set (the secondary measurements of the default run)
    -- as many steps as fill that many seconds, so that the clock sampler
    (one sample per 100 ms) sees the region.  Returns the per-step CUDA-event
    times, the clock summary and the number of timed steps."""
    import torch
    steps = args.steps
    if getattr(args, "min_timed_s", 0):
        per = max(1e-3, statistics.median(time_events(fn, 3, stream)))
        steps = max(steps, int(math.ceil(args.min_timed_s * 1e3 / per)))
    with Clocks(torch.cuda.current_device()) as clk:
        ts = time_events(fn, steps, stream)
    return ts, clk.summary(), steps


def l2_flusher():
    import torch
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        buf.zero_()
    return flush


# ---------------------------------------------------------------- workloads

def kstats(L, ctx, name, reset=True):
    ms, n = C.c_double(), C.c_uint64()
    L.check(L.lib().chai_cuda_kernel_stats(ctx, name.encode(), C.byref(ms), C.byref(n), 1 if reset else 0), ctx)
    return ms.value, n.value


def traffic(name):
    """Per-launch DRAM bytes from the committed ncu summary (profiles/ncu_traffic.json)."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if p.exists():
        return json.loads(p.read_text()).get(name)
    return None


def issue_roofline(kernel_ms, units, key, kernel):
    """Roofline of an instruction-issue-bound kernel (the fused MC trace: no
    HBM traffic, Philox integer multiplies and transcendental math):
    achieved = warp instructions per launch (units x the per-unit count from
    the committed ncu summary, smsp__inst_executed.sum) / launch time; peak =
    148 SMs x 4 schedulers x one warp instruction per clock at the maximum SM
    clock of MEASURED_PEAKS.json."""
    P, kind = peaks()
    per_unit = traffic(key)
    if not kernel_ms or not per_unit:
        return None
    mhz = P.get("sm_max_mhz", 1965.0)
    peak = 148 * 4 * mhz * 1e6 / 1e12          # warp instructions per second, in T/s
    ach = units * per_unit / (kernel_ms * 1e-3) / 1e12
    return {"bound": "issue", "achieved": ach, "peak": peak, "unit": "Twarp-inst/s", "frac": ach / peak,
            "traffic": None, "peak_source": "148 SMs x 4 issue slots x %s max SM clock (%s)" % (mhz, kind),
            "kernel": kernel, "kernel_ms": kernel_ms, "warp_inst_per_unit": per_unit}


GEMM_PREC = {"fp32": 0, "tf32": 1, "bf16": 2, "bf16x3": 3, "bf16x6": 4, "fp8": 5}
TENSOR_MULT = {0: 0, 1: 1, 2: 1, 3: 3, 4: 6, 5: 1}


def gemm_operands(L, ctx, n, dist):
    """f32 n x n operands from the library's own Philox fill (chai layout):
    uniform[-1, 1) with seeds 1, 2, or N(0, 1) (Box-Muller) with seeds 3, 4."""
    import torch
    out = []
    for seed in ((1, 2) if dist == "uniform" else (3, 4)):
        t = torch.empty((n, n), device="cuda", dtype=torch.float32)
        if dist == "uniform":
            rd = L.chai_rng_desc(1230, 4, 0, 4, seed, n, n, 1, 1, -1.0, 1.0)
        else:
            rd = L.chai_rng_desc(1230, 4, 1, 4, seed, n, n, 1, 0, 0.0, 1.0)
        L.check(L.lib().chai_cuda_rng_fill(ctx, C.byref(rd), C.c_void_p(t.data_ptr())), ctx)
        if dist == "normal":
            # chai's Box-Muller gives +-inf for the rare u = 0 draws (about one
            # in 2^25); the precision sweep needs finite operands
            t.nan_to_num_(nan=0.0, posinf=0.0, neginf=0.0)
        out.append(t)
    return out


def gemm_error(A, B, Cm, samples=4096, seed=0):
    """Error of C against the FP64 product on `samples` random entries (FP64
    dot products on the GPU): max |C - C64| / (|A| |B|)_ij (componentwise-bound
    normalised) and max |C - C64| / |C64|."""
    import torch
    n_m, n_n = Cm.shape
    g = torch.Generator(device="cuda").manual_seed(seed)
    rows = torch.randint(0, n_m, (samples,), device="cuda", generator=g)
    cols = torch.randint(0, n_n, (samples,), device="cuda", generator=g)
    num, bnd = [], []
    for c0 in range(0, samples, 512):
        r, c = rows[c0:c0 + 512], cols[c0:c0 + 512]
        a = A[r].double()
        b = B[:, c].double().t()
        num.append((a * b).sum(1))
        bnd.append((a.abs() * b.abs()).sum(1))
    c64 = torch.cat(num)
    bound = torch.cat(bnd)
    got = Cm[rows, cols].double()
    err = (got - c64).abs()
    ok = torch.isfinite(got)
    return {"max_err_normalized": float((err / bound.clamp_min(1e-300)).max()),
            "max_rel_err": float((err / c64.abs().clamp_min(1e-300)).max()),
            "finite": bool(ok.all()), "error_samples": samples}


def run_gemm(args, L, ctx, stream):
    import torch
    n = args.size or 16384
    prec = GEMM_PREC[args.precision]
    A, B = gemm_operands(L, ctx, n, "uniform")
    Cm = torch.empty((n, n), device="cuda", dtype=torch.float32)
    d = L.chai_gemm_desc(prec, 0, 0, 0, n, n, n, A.data_ptr(), n, B.data_ptr(), n, Cm.data_ptr(), n, 1.0, 0.0, 1,
                         0, 0, 0)

    def step():
        L.check(L.lib().chai_cuda_gemm(ctx, C.byref(d)), ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "gemm_tc")
    flops = 2.0 * n ** 3
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    k_ms, k_n = kstats(L, ctx, "gemm_tc")
    kern_ms = k_ms / k_n if k_n else None
    err = gemm_error(A, B, Cm)
    # e2e through the public entry points: pinned host A, B in, C out each step
    Ah = A.cpu().pin_memory()
    Bh = B.cpu().pin_memory()
    Ch = torch.empty((n, n), dtype=torch.float32).pin_memory()
    # e2e: the host-operand GEMM entry point -- B uploaded once, A streamed up
    # and C streamed back in row blocks, the copies overlapped with the GEMMs
    de = L.chai_gemm_desc(prec, 0, 0, 0, n, n, n, Ah.data_ptr(), n, Bh.data_ptr(), n, Ch.data_ptr(), n, 1.0, 0.0,
                          1, 0, 0, 0)
    del A, B, Cm
    torch.cuda.empty_cache()

    def e2e():
        L.check(L.lib().chai_cuda_gemm_host(ctx, C.byref(de), 0), ctx)

    e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    esteps = max(1, min(args.steps, 5))
    for _ in range(esteps):
        e2e()
    torch.cuda.synchronize()
    e_ms = (time.perf_counter() - t0) * 1e3 / esteps
    P, kind = peaks()
    tensor_flops = flops * TENSOR_MULT[prec]
    roof = None
    # the CTA-pair kernel (cta_group::2) runs every non-fp8 GEMM with M > 128
    # under the default 256-row tile; fp8 stays on the one-CTA kernel
    kname = "pair" if prec != 5 and n > 128 else "tc"
    if prec and kern_ms:
        achieved = tensor_flops / (kern_ms * 1e-3) / 1e12
        # the tensor pipe's dense rate: tf32 half of bf16, fp8 twice bf16
        rate = {1: 0.5, 5: 2.0}.get(prec, 1.0)
        peak = P["bf16_tflops"] * rate
        src = "%s (bf16 dense, burst)" % kind if rate == 1.0 else \
            "%s bf16 dense burst x %g (the %s rate)" % (kind, rate, args.precision)
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic("gemm_%s_%s_%d" % (kname, args.precision, n)),
                "peak_source": src, "kernel": "chai_gemm_" + kname,
                "kernel_ms": kern_ms, "algorithmic_flops": tensor_flops}
    return {
        "metric": "GEMM TFLOP/s at err vs FP32", "unit": "TFLOP/s", "value": flops / (ms * 1e-3) / 1e12,
        "ms_per_step": ms, "dtype": args.precision, "higher_is_better": True,
        "config": {"workload": "square GEMM M=N=K=%d, f32 operands uniform[-1,1) (chai Philox seeds 1,2), %s"
                   % (n, args.precision), "m": n, "n": n, "k": n,
                   "l2": "operands (%d MiB each) larger than L2" % (n * n * 4 >> 20),
                   "includes": "operand split/transposition prepass + tcgen05 GEMM", "error_vs_fp64": err,
                   "e2e_path": "chai_cuda_gemm_host: pinned host A, B, C; B uploaded, A and C streamed in row "
                               "blocks with the copies overlapped with the block GEMMs"},
        "e2e": {"value": flops / (e_ms * 1e-3) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 2 * n * n * 4,
                "d2h_bytes_per_step": n * n * 4},
        "roofline": roof, "clocks": clk, "steps": steps, "gpu_launches": steps * {0: 1, 5: 6}.get(prec, 3),
    }


def gemm_sweep(args, L, ctx, stream, path):
    """The GEMM precision sweep: M = N = K in {1024 .. 16384}, uniform[-1, 1)
    and N(0, 1) operands, every arithmetic; time (CUDA events, median of 3
    after a warm-up) and error against FP64 per shape.  Written to `path`."""
    import torch
    rows = []
    for n in (1024, 2048, 4096, 8192, 16384):
        for dist in ("uniform", "normal"):
            A, B = gemm_operands(L, ctx, n, dist)
            Cm = torch.empty((n, n), device="cuda", dtype=torch.float32)
            for name in ("fp32", "tf32", "bf16", "bf16x3", "bf16x6", "fp8"):
                if name == "fp32" and n > 8192 and dist == "normal":
                    continue
                d = L.chai_gemm_desc(GEMM_PREC[name], 0, 0, 0, n, n, n, A.data_ptr(), n, B.data_ptr(), n,
                                     Cm.data_ptr(), n, 1.0, 0.0, 1, 0, 0, 0)

                def step():
                    L.check(L.lib().chai_cuda_gemm(ctx, C.byref(d)), ctx)
                step()
                ts = time_events(step, 3, stream)
                ms = statistics.median(ts)
                row = {"n": n, "dist": dist, "precision": name, "ms": ms,
                       "tflops": 2.0 * n ** 3 / (ms * 1e-3) / 1e12}
                row.update(gemm_error(A, B, Cm, samples=2048))
                rows.append(row)
                print(json.dumps(row), file=sys.stderr)
            del A, B, Cm
            torch.cuda.empty_cache()
    with open(path, "w") as f:
        json.dump(rows, f, indent=1)


def mc_expr(ch, g, W, H):
    f = np.float32
    return ch.mean(ch.max(f(100) * ch.exp(f(0.05 - 0.5 * 0.2 * 0.2) + f(0.2) * ch.rng_normal_make(g, W, H))
                          - f(100), f(0)))


def record(ch, build):
    ch._Client.pending = []
    out = build()
    stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    ch._Client.pending = []
    return stmts, out


def run_mc(args, L, ctx, stream):
    import torch
    import chai_b200.api as ch
    W, H = 8192, 16384                 # 2^27 normals from 2^26 Box-Muller pairs
    dev = ch.vm()
    n = W * H
    stmts, p = record(ch, lambda: ch.Arrayf32(mc_expr(ch, ch.RNGf32(ch.RNG_PHILOX, 42), W, H)))
    bid = 77001
    desc, keep = ch.build_desc(stmts)
    barr = (L.chai_buffer_binding * 1)(L.chai_buffer_binding(p.var, 4, 1, 1, 1, 0, bid))

    def step():
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr, 1), dev.ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "trace")
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    k_ms, k_n = kstats(L, ctx, "trace")

    def e2e():
        return float(ch.Arrayf32(mc_expr(ch, ch.RNGf32(ch.RNG_PHILOX, 42), W, H)).read_scalar())

    payoff = e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps)):
        payoff = e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / max(1, args.steps)
    roof = issue_roofline(k_ms / k_n if k_n else None, n, "trace_mc_warp_inst_per_normal",
                          "chai_group (MC trace, RNG in registers)")
    return {
        "metric": "trace throughput (MC: Philox normals -> exp -> mean)", "unit": "Gnormals/s",
        "value": n / (ms * 1e-3) / 1e9, "ms_per_step": ms, "dtype": "f32", "higher_is_better": True,
        "config": {"workload": "Monte Carlo trace, 2^27 Philox4x32-10 Box-Muller normals, fused", "normals": n,
                   "payoff": payoff, "l2": "no HBM inputs (RNG in registers)",
                   "kernel_ms": (k_ms / k_n) if k_n else None},
        "e2e": {"value": n / (e_ms * 1e-3) / 1e9, "unit": "Gnormals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 16},
        "roofline": roof, "clocks": clk, "steps": steps, "gpu_launches": steps * 2,
    }


C1_N = 512


def c1_expr(ch, g, n=C1_N):
    """The C1 trace: A, B uniform[-1, 1) from one chai Philox generator (seed 0,
    the second fill continues the first's counters), C = matmul(A, B),
    s = sum(C * C)."""
    a = ch.Arrayf32(ch.rng_uniform_make(g, n, n, 1, -1.0, 1.0))
    b = ch.Arrayf32(ch.rng_uniform_make(g, n, n, 1, -1.0, 1.0))
    c = ch.Arrayf32(ch.matmul(a, b))
    return ch.sum(c * c)


def count_launches(step):
    """Kernels one call of `step` launches (torch profiler, outside any timed
    region); None where the profiler cannot see CUDA activity."""
    import torch
    try:
        from torch.profiler import ProfilerActivity, profile
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            step()
            torch.cuda.synchronize()
        return sum(1 for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA
                   and "memcpy" not in e.name.lower() and "memset" not in e.name.lower())
    except Exception:
        return None


def run_c1(args, L, ctx, stream):
    """C1: 512^3 matmul + sum(C * C) as one traced program (latency-bound at
    this size: the line reports microseconds per evaluation beside TFLOP/s)."""
    import torch
    import chai_b200.api as ch
    n = C1_N
    # the evaluation a user's context runs: kernel timing off, so repeated
    # evaluations replay as one captured CUDA graph (PlanGraph=1 says so
    # explicitly; this bench's main context times kernels for the rooflines)
    dev = ch.Device(config=" ".join(x for x in (args.config, "PlanGraph=1") if x))
    try:
        L.check(L.lib().chai_cuda_set_stream(dev.ctx, C.c_void_p(stream.cuda_stream)), dev.ctx)
        out = _run_c1(args, L, ch, dev, n, stream)
    finally:
        dev.close()
    out["roofline"] = _c1_gemm_roofline(L, ch, ctx, n)
    return out


def _c1_gemm_roofline(L, ch, ctx, n):
    """The C1 line's roofline: its dominant kernel, the bf16x3 tcgen05 GEMM of
    the 512^3 product, timed with CUDA events on the bench's main context
    (kernel timing on) over a few evaluations of the same trace.  Tensor work:
    three bf16 products, 3 x 2 n^3.  At this size the GEMM is latency-bound,
    so the fraction is small by construction; the line's time is the six
    dependent launches of one evaluation."""
    import torch
    try:
        stmts, s_arr = record(ch, lambda: ch.Arrayf32(c1_expr(ch, ch.RNGf32(ch.RNG_PHILOX, 0))))
        desc, keep = ch.build_desc(stmts)
        barr = (L.chai_buffer_binding * 1)(L.chai_buffer_binding(s_arr.var, 4, 1, 1, 1, 0, 77202))
        for _ in range(3):
            L.check(L.lib().chai_cuda_evaluate(ctx, C.byref(desc), barr, 1), ctx)
        torch.cuda.synchronize()
        kstats(L, ctx, "gemm_tc")
        for _ in range(10):
            L.check(L.lib().chai_cuda_evaluate(ctx, C.byref(desc), barr, 1), ctx)
        torch.cuda.synchronize()
        g_ms, g_n = kstats(L, ctx, "gemm_tc")
        L.lib().chai_cuda_release(ctx, 77202)
        if not g_n:
            return None
        P, kind = peaks()
        kern_ms = g_ms / g_n
        flops = 3 * 2.0 * n ** 3
        ach = flops / (kern_ms * 1e-3) / 1e12
        return {"bound": "tensor", "achieved": ach, "peak": P["bf16_tflops"], "unit": "TFLOP/s",
                "frac": ach / P["bf16_tflops"], "traffic": None, "peak_source": "%s (bf16 dense, burst)" % kind,
                "kernel": "chai_gemm_tc_kernel (bf16x3, 512^3)", "kernel_ms": kern_ms, "algorithmic_flops": flops,
                "note": "latency-bound: 32 one-CTA 128x64 tiles, 8 K chunks each"}
    except Exception:
        return None


def _run_c1(args, L, ch, dev, n, stream):
    import torch
    flops = 2.0 * n ** 3 + 2.0 * n * n
    stmts, s_arr = record(ch, lambda: ch.Arrayf32(c1_expr(ch, ch.RNGf32(ch.RNG_PHILOX, 0))))
    bid = 77201
    desc, keep = ch.build_desc(stmts)
    barr = (L.chai_buffer_binding * 1)(L.chai_buffer_binding(s_arr.var, 4, 1, 1, 1, 0, bid))

    def step():
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr, 1), dev.ctx)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    per_step = count_launches(step)
    # e2e: A and B from pinned host memory through make2 every evaluation,
    # the scalar read back
    rng = np.random.default_rng(0)
    Ah = torch.from_numpy(rng.uniform(-1, 1, (n, n)).astype(np.float32)).pin_memory().numpy()
    Bh = torch.from_numpy(rng.uniform(-1, 1, (n, n)).astype(np.float32)).pin_memory().numpy()

    def e2e():
        c = ch.Arrayf32(ch.matmul(ch.make2(Ah), ch.make2(Bh)))
        return float(ch.Arrayf32(ch.sum(c * c)).read_scalar())

    for _ in range(3):
        e2e()
    torch.cuda.synchronize()
    reps = max(5, args.steps)
    t0 = time.perf_counter()
    for _ in range(reps):
        sv = e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / reps
    return {
        "metric": "C1 trace TFLOP/s (512^3 matmul + sum(C*C))", "unit": "TFLOP/s",
        "value": flops / (ms * 1e-3) / 1e12, "ms_per_step": ms, "dtype": "f32", "higher_is_better": True,
        "config": {"workload": "C1: A, B = chai Philox uniform[-1,1) 512x512 (seed 0), C = matmul(A, B), "
                               "s = sum(C*C), one traced evaluation (plan replay)",
                   "us_per_evaluation": ms * 1e3, "e2e_us_per_evaluation": e_ms * 1e3, "s_e2e": sv,
                   "gemm_precision": "context default", "l2": "inputs generated in the trace (no HBM inputs)",
                   "replay": "captured CUDA graph of the plan (PlanGraph=1); e2e: fresh uploads each "
                             "evaluation, plain plan replay"},
        "e2e": {"value": flops / (e_ms * 1e-3) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 2 * n * n * 4,
                "d2h_bytes_per_step": 4},
        "roofline": None, "clocks": clk, "steps": steps,
        "gpu_launches": (per_step * steps) if per_step is not None else steps * 6,
    }


def run_mc_hbm(args, L, ctx, stream):
    """The materialised Monte Carlo variant: Z (2^27 f32 normals, 512 MiB)
    already in HBM, payoff = mean(max(100 exp(0.03 + 0.2 Z) - 100, 0)) as one
    fused trace reading it once (4 bytes per element)."""
    import torch
    import chai_b200.api as ch
    W, H = 8192, 16384
    n = W * H
    dev = ch.vm()
    z = torch.empty(n, device="cuda", dtype=torch.float32)
    rd = L.chai_rng_desc(1230, 4, 1, 4, 42, W, H, 1, 0, 0.0, 1.0)
    L.check(L.lib().chai_cuda_rng_fill(ctx, C.byref(rd), C.c_void_p(z.data_ptr())), ctx)
    z.nan_to_num_(nan=0.0, posinf=0.0, neginf=0.0)      # the rare u = 0 draws
    zid, pid = 77101, 77102
    L.check(L.lib().chai_cuda_buffer_wrap(ctx, zid, C.c_void_p(z.data_ptr()), n * 4), ctx)
    ch._Client.pending = []
    z_var = next(ch._Client.vars)
    Z = ch._Raw([ch._bc(L.BC_VARIABLE, z_var, 0)], L.F32, W, H)
    f = np.float32
    P = ch.Arrayf32(ch.mean(ch.max(f(100) * ch.exp(f(0.05 - 0.5 * 0.2 * 0.2) + f(0.2) * Z) - f(100), f(0))))
    stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    ch._Client.pending = []
    desc, keep = ch.build_desc(stmts)
    barr = (L.chai_buffer_binding * 2)(L.chai_buffer_binding(z_var, 4, W, H, 1, 0, zid),
                                       L.chai_buffer_binding(P.var, 4, 1, 1, 1, 0, pid))

    def step():
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr, 2), dev.ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "trace")
    # Z (512 MiB) is four times L2: streamed from HBM each step without a flush
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    k_ms, k_n = kstats(L, ctx, "trace")
    kern_ms = k_ms / k_n if k_n else None
    nbytes = 4 * n
    P_, kind = peaks()
    roof = None
    if kern_ms:
        ach = nbytes / (kern_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": P_["hbm_gbs"], "unit": "GB/s", "frac": ach / P_["hbm_gbs"],
                "traffic": traffic("trace_mc_hbm"), "peak_source": "%s (copy)" % kind,
                "kernel": "chai_group (MC over Z in HBM)", "kernel_ms": kern_ms, "algorithmic_bytes": nbytes}
    # e2e: Z from pinned host memory each step, payoff read back
    zh = z.cpu().pin_memory()
    ze = 77103
    L.check(L.lib().chai_cuda_buffer_alloc(ctx, ze, n * 4), ctx)
    barr2 = (L.chai_buffer_binding * 2)(L.chai_buffer_binding(z_var, 4, W, H, 1, 0, ze),
                                        L.chai_buffer_binding(P.var, 4, 1, 1, 1, 0, pid))
    out = (C.c_float * 1)()

    def e2e():
        L.check(L.lib().chai_cuda_upload(ctx, ze, C.c_void_p(zh.data_ptr()), n * 4), ctx)
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr2, 2), dev.ctx)
        L.check(L.lib().chai_cuda_readback(ctx, pid, out, 4), ctx)

    e2e()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 5))):
        e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / max(1, min(args.steps, 5))
    return {
        "metric": "trace HBM GB/s", "unit": "GB/s", "value": nbytes / (ms * 1e-3) / 1e9, "ms_per_step": ms,
        "dtype": "f32", "higher_is_better": True,
        "config": {"workload": "Monte Carlo payoff over 2^27 f32 normals already in HBM (materialised Z), fused",
                   "normals": n, "payoff": float(out[0]), "l2": "Z (512 MiB) larger than L2, no flush"},
        "e2e": {"value": nbytes / (e_ms * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": 4},
        "roofline": roof, "clocks": clk, "steps": steps, "gpu_launches": steps * 2,
    }


def kirsch_expr(ch, A, W, H):
    f = np.float32
    X, Y = ch.index_f32(0, W, H), ch.index_f32(1, W, H)
    one = f(1)
    nb = [ch.gather2_floor(A, X - one, Y - one), ch.gather2_floor(A, X, Y - one),
          ch.gather2_floor(A, X + one, Y - one), ch.gather2_floor(A, X + one, Y),
          ch.gather2_floor(A, X + one, Y + one), ch.gather2_floor(A, X, Y + one),
          ch.gather2_floor(A, X - one, Y + one), ch.gather2_floor(A, X - one, Y)]
    total = nb[0] + nb[1] + nb[2] + nb[3] + nb[4] + nb[5] + nb[6] + nb[7]
    r = [f(8) * ((nb[k] + nb[(k + 1) % 8]) + nb[(k + 2) % 8]) - f(3) * total for k in range(8)]
    return ch.max(ch.max(ch.max(r[0], r[1]), ch.max(r[2], r[3])), ch.max(ch.max(r[4], r[5]), ch.max(r[6], r[7])))


def run_kirsch(args, L, ctx, stream):
    import torch
    import chai_b200.api as ch
    W = H = args.size or 8192
    dev = ch.vm()
    img = torch.empty((H, W), device="cuda", dtype=torch.float32)
    rd = L.chai_rng_desc(1230, 4, 0, 4, 5, W, H, 1, 1, 0.0, 1.0)
    L.check(L.lib().chai_cuda_rng_fill(ctx, C.byref(rd), C.c_void_p(img.data_ptr())), ctx)
    out = torch.empty_like(img)
    in_id, out_id = 88001, 88002
    L.check(L.lib().chai_cuda_buffer_wrap(ctx, in_id, C.c_void_p(img.data_ptr()), img.numel() * 4), ctx)
    L.check(L.lib().chai_cuda_buffer_wrap(ctx, out_id, C.c_void_p(out.data_ptr()), out.numel() * 4), ctx)

    def build():
        A = ch._ARR[4](_raw=([ch._bc(0, 0), ], W, H, 1))
        return A
    # trace: A bound as an input variable, K bound as an output variable
    ch._Client.pending = []
    a_var = next(ch._Client.vars)
    A = ch._Raw([ch._bc(1, a_var, 0)], 4, W, H)
    K = ch.Arrayf32(kirsch_expr(ch, A, W, H))
    stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    ch._Client.pending = []
    desc, keep = ch.build_desc(stmts)
    barr = (L.chai_buffer_binding * 2)(L.chai_buffer_binding(a_var, 4, W, H, 1, 0, in_id),
                                       L.chai_buffer_binding(K.var, 4, W, H, 1, 0, out_id))

    def step():
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr, 2), dev.ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "trace")
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    k_ms, k_n = kstats(L, ctx, "trace")
    nbytes = 2 * 4 * W * H
    # e2e: host image in (pinned), edge map out, through the public API
    hin = img.cpu().pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    e_in, e_out = 88003, 88004
    L.check(L.lib().chai_cuda_buffer_alloc(ctx, e_in, W * H * 4), ctx)
    barr2 = (L.chai_buffer_binding * 2)(L.chai_buffer_binding(a_var, 4, W, H, 1, 0, e_in),
                                        L.chai_buffer_binding(K.var, 4, W, H, 1, 0, e_out))

    def e2e():
        L.check(L.lib().chai_cuda_upload(ctx, e_in, C.c_void_p(hin.data_ptr()), W * H * 4), ctx)
        L.check(L.lib().chai_cuda_evaluate(dev.ctx, C.byref(desc), barr2, 2), dev.ctx)
        L.check(L.lib().chai_cuda_readback(ctx, e_out, C.c_void_p(hout.data_ptr()), W * H * 4), ctx)

    e2e()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 5))):
        e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / max(1, min(args.steps, 5))
    P, kind = peaks()
    kern_ms = k_ms / k_n if k_n else None
    roof = None
    if kern_ms:
        ach = nbytes / (kern_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": P["hbm_gbs"], "unit": "GB/s", "frac": ach / P["hbm_gbs"],
                "traffic": traffic("trace_kirsch_%d" % W), "peak_source": "%s (copy)" % kind,
                "kernel": "chai_group (Kirsch trace)", "kernel_ms": kern_ms, "algorithmic_bytes": nbytes}
    return {
        "metric": "trace HBM GB/s", "unit": "GB/s", "value": nbytes / (ms * 1e-3) / 1e9, "ms_per_step": ms,
        "dtype": "f32", "higher_is_better": True,
        "config": {"workload": "Kirsch 8-direction compass filter via gather2_floor, %dx%d f32 uniform[0,1)"
                   % (W, H), "l2": "image (%d MiB) larger than L2" % (W * H * 4 >> 20)},
        "e2e": {"value": nbytes / (e_ms * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": W * H * 4,
                "d2h_bytes_per_step": W * H * 4},
        "roofline": roof, "clocks": clk, "steps": steps, "gpu_launches": steps,
    }


def run_gemv(args, L, ctx, stream):
    import torch
    m = n = args.size or 8192
    dt = torch.float64 if args.precision == "f64" else torch.float32
    prec = 8 if dt == torch.float64 else 4
    eb = 8 if prec == 8 else 4
    A = torch.rand((m, n), device="cuda", dtype=dt) * 2 - 1
    x = torch.rand(n, device="cuda", dtype=dt) * 2 - 1
    y = torch.empty(m, device="cuda", dtype=dt)

    def step():
        L.check(L.lib().chai_cuda_gemv(ctx, prec, 0, m, n, 1.0, C.c_void_p(A.data_ptr()), n,
                                       C.c_void_p(x.data_ptr()), 0.0, C.c_void_p(y.data_ptr())), ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "gemv")
    # A (>= 256 MiB at the default size) is at least twice L2: each step
    # streams it from HBM without a flush (a written flush buffer would leave
    # dirty L2 lines whose write-back the next step would pay for)
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    k_ms, k_n = kstats(L, ctx, "gemv")
    nbytes = (m * n + m + n) * eb
    P, kind = peaks()
    kern_ms = k_ms / k_n if k_n else ms
    ach = nbytes / (kern_ms * 1e-3) / 1e9
    return {
        "metric": "GEMV GB/s", "unit": "GB/s", "value": nbytes / (ms * 1e-3) / 1e9, "ms_per_step": ms,
        "dtype": "f64" if prec == 8 else "f32", "higher_is_better": True,
        "config": {"workload": "GEMV y = A x, %dx%d %s" % (m, n, "f64" if prec == 8 else "f32"),
                   "l2": "A (%d MiB) larger than L2, no flush" % (m * n * eb >> 20)},
        "e2e": None,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": P["hbm_gbs"], "unit": "GB/s",
                     "frac": ach / P["hbm_gbs"], "traffic": traffic("gemv_%d" % m), "peak_source": kind,
                     "kernel": "chai_gemv_n", "kernel_ms": kern_ms, "algorithmic_bytes": nbytes},
        "clocks": clk, "steps": steps, "gpu_launches": steps,
    }


def many_lengths(n=64, seed=7):
    """Trace lengths log-uniform in [2^12, 2^22], rounded to multiples of 4."""
    rng = np.random.default_rng(seed)
    return [int(4 * round(2.0 ** u / 4)) for u in rng.uniform(12, 22, n)]


def run_mc_many(args, L, ctx, stream):
    import torch
    import chai_b200.api as ch
    Ls = many_lengths()
    total = sum(Ls)

    def mc1(seed, W):
        return ch.Arrayf32(mc_expr(ch, ch.RNGf32(ch.RNG_PHILOX, seed), W, 1))
    traces = [ch.record(lambda s=s, W=W: mc1(42 + s, W))[0] for s, W in enumerate(Ls)]
    descs = []
    ptrs = (C.POINTER(L.chai_trace_desc) * len(traces))()
    for i, st in enumerate(traces):
        d, k = ch.build_desc(st)
        descs.append((d, k))
        ptrs[i] = C.pointer(d)
    res = (C.c_double * len(traces))()

    def step():
        L.check(L.lib().chai_cuda_evaluate_many(ctx, ptrs, len(traces), res), ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "many")
    steps = args.steps
    if getattr(args, "min_timed_s", 0):
        t0 = time.perf_counter()
        for _ in range(3):
            step()
        per = max(1e-3, (time.perf_counter() - t0) * 1e3 / 3)
        steps = max(steps, int(math.ceil(args.min_timed_s * 1e3 / per)))
    with Clocks(torch.cuda.current_device()) as clk:
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        wall = (time.perf_counter() - t0) * 1e3 / steps
    clk = clk.summary()
    k_ms, k_n = kstats(L, ctx, "many")
    kern = k_ms / k_n if k_n else wall

    def e2e():      # record 64 traces through the front end and evaluate them
        tr = [ch.record(lambda s=s, W=W: mc1(42 + s, W))[0] for s, W in enumerate(Ls)]
        return ch.evaluate_many(tr)
    e2e()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 5))):
        e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / max(1, min(args.steps, 5))
    return {
        "metric": "trace throughput (64 uneven MC traces, one persistent launch)", "unit": "Gnormals/s",
        "value": total / (kern * 1e-3) / 1e9, "ms_per_step": kern, "dtype": "f32", "higher_is_better": True,
        "config": {"workload": "64 MC traces, lengths log-uniform in [2^12, 2^22] (seed 7), one persistent kernel "
                               "+ combine captured in a CUDA graph", "normals": total,
                   "host_ms_per_call": wall, "l2": "no HBM inputs (RNG in registers)"},
        "e2e": {"value": total / (e_ms * 1e-3) / 1e9, "unit": "Gnormals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8 * len(Ls)},
        # issue roofline of chai_many (warp instructions per normal from
        # profiles/many_traces_mc_many.md); the timed region also holds the
        # combine (about 3 us of the step)
        "roofline": issue_roofline(kern if k_n else None, total, "trace_many_warp_inst_per_normal",
                                   "chai_many (+ chai_many_combine in the timed graph)"),
        "clocks": clk, "steps": steps, "gpu_launches": steps * 2,
    }


def grouped_shapes(count=4096, seed=11):
    """M, N, K uniform over the multiples of 8 in [32, 512] (seed 11)."""
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.integers(4, 65, 3) * 8) for _ in range(count)]


def run_grouped(args, L, ctx, stream):
    import torch
    shapes = grouped_shapes(args.size or 4096)
    prec = GEMM_PREC[args.precision] if args.precision in GEMM_PREC else 3
    if prec in (0, 1):
        prec = 3
    g = torch.Generator(device="cuda").manual_seed(3)
    sa = sum(m * k for m, n, k in shapes)
    sb = sum(k * n for m, n, k in shapes)
    sc = sum(m * n for m, n, k in shapes)
    A = torch.rand(sa, device="cuda", generator=g) * 2 - 1
    B = torch.rand(sb, device="cuda", generator=g) * 2 - 1
    Cm = torch.empty(sc, device="cuda")
    arr = (L.chai_gemm_problem * len(shapes))()
    oa = ob = oc = 0
    for i, (m, n, k) in enumerate(shapes):
        arr[i] = L.chai_gemm_problem(m, n, k, 0, A.data_ptr() + 4 * oa, B.data_ptr() + 4 * ob, Cm.data_ptr() + 4 * oc)
        oa += m * k
        ob += k * n
        oc += m * n
    flops = sum(2.0 * m * n * k for m, n, k in shapes)

    def step():
        L.check(L.lib().chai_cuda_gemm_grouped(ctx, prec, arr, len(shapes)), ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kstats(L, ctx, "gemm_grouped")
    ts, clk, steps = timed_region(step, args, stream)
    ms = sum(ts) / len(ts)
    k_ms, k_n = kstats(L, ctx, "gemm_grouped")
    kern = k_ms / k_n if k_n else ms
    # e2e: host operands in, results out
    Ah, Bh = A.cpu().pin_memory(), B.cpu().pin_memory()
    Ch = torch.empty(sc).pin_memory()

    def e2e():
        A.copy_(Ah, non_blocking=True)
        B.copy_(Bh, non_blocking=True)
        step()
        Ch.copy_(Cm, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    e2e()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 5))):
        e2e()
    e_ms = (time.perf_counter() - t0) * 1e3 / max(1, min(args.steps, 5))
    P, kind = peaks()
    tensor_mult = TENSOR_MULT[prec]
    ach = flops * tensor_mult / (kern * 1e-3) / 1e12
    # Which roof binds: these problems (mean M = N = K = 272) sit below the
    # machine balance, so the f32 operands read once and C written once
    # (algorithmic bytes) take longer at HBM peak than the tensor work at
    # tensor peak; the line reports against the binding roof and gives both.
    alg_bytes = 4 * (sa + sb + sc)
    t_hbm = alg_bytes / (P["hbm_gbs"] * 1e9)
    t_tc = flops * tensor_mult / (P["bf16_tflops"] * 1e12)
    gbs = alg_bytes / (kern * 1e-3) / 1e9
    common = {"traffic": traffic("gemm_grouped"), "peak_source": kind, "kernel_ms": kern,
              "kernel": "chai_gemm_fused_pair (grouped, operands split in-kernel, 256x256 CTA-pair tiles)",
              "algorithmic_bytes": alg_bytes, "algorithmic_tensor_flops": flops * tensor_mult,
              "tensor_frac": ach / P["bf16_tflops"], "hbm_frac": gbs / P["hbm_gbs"],
              "floor_ms": {"hbm": t_hbm * 1e3, "tensor": t_tc * 1e3}}
    if t_hbm >= t_tc:
        roof = dict({"bound": "hbm", "achieved": gbs, "peak": P["hbm_gbs"], "unit": "GB/s",
                     "frac": gbs / P["hbm_gbs"]}, **common)
    else:
        roof = dict({"bound": "tensor", "achieved": ach, "peak": P["bf16_tflops"], "unit": "TFLOP/s",
                     "frac": ach / P["bf16_tflops"]}, **common)
    return {
        "metric": "GEMM TFLOP/s at err vs FP32", "unit": "TFLOP/s", "value": flops / (ms * 1e-3) / 1e12,
        "ms_per_step": ms, "dtype": args.precision if prec != 3 else "bf16x3", "higher_is_better": True,
        "config": {"workload": "%d grouped f32 GEMMs, M,N,K multiples of 8 in [32,512] (seed 11), one persistent "
                               "tcgen05 launch" % len(shapes), "problems": len(shapes), "useful_gflop": flops / 1e9},
        "e2e": {"value": flops / (e_ms * 1e-3) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 4 * (sa + sb),
                "d2h_bytes_per_step": 4 * sc},
        "roofline": roof, "clocks": clk, "steps": steps,
        # one persistent GEMM launch per call (the tile records are built once
        # per problem array, in the warm-up)
        "gpu_launches": steps,
    }


def run_tuner(args, L, ctx, stream):
    """Learned tuner: exhaustive sweeps over 2000 training keys and 200 held-out
    keys (M, N, K log-uniform in [64, 16384], seed 13, fp32 via bf16x3 and bf16
    GEMM plus f32 GEMV), MLP trained on the GPU, then each held-out key tuned
    twice from cold: learned (rank all configurations, time the top k) and
    exhaustive (time all).  Quality is judged on the held-out key's own sweep."""
    import torch
    from chai_b200 import tuner as T
    n_train = args.size or 2000
    keys = T.shapes(n_train + 200, seed=13)
    train_keys, held_keys = keys[:n_train], keys[n_train:]
    data, sweep_s = T.collect(ctx, train_keys, log=lambda m: print(m, file=sys.stderr))
    held, _ = T.collect(ctx, held_keys, repeats=3)
    samples = [(k, c) for k, cs in data for c in cs if c.measured_us < 1e29]
    t0 = time.perf_counter()
    loss = T.train(ctx, samples, epochs=args.steps if args.steps > 100 else 4000, lr=1e-3, seed=1)
    train_s = time.perf_counter() - t0
    import chai_b200.api as ch
    gm = lambda v: float(np.exp(np.mean(np.log(v)))) if len(v) else None
    by_k = {}
    with tempfile.TemporaryDirectory() as td, Clocks(torch.cuda.current_device()) as clk:
        db = os.path.join(td, "tune.db")
        L.check(L.lib().chai_cuda_tune_db_save(ctx, db.encode()), ctx)
        if getattr(args, "save_db", False):     # the committed cost model the default run evaluates
            TUNER_DB.parent.mkdir(exist_ok=True)
            L.check(L.lib().chai_cuda_tune_db_save(ctx, str(TUNER_DB).encode()), ctx)
        for k in (1, 2, 3):     # a fresh context per k: cold DB, the trained weights
            dev = ch.Device(config="TuneDB=%s TopK=%d" % (db, k))
            try:
                r = T.evaluate(dev.ctx, held)
            finally:
                dev.close()
            by_k[k] = r
    rows = by_k[3]
    topk = {k: {"pick_vs_best_geomean": gm(np.array([x["best_us"] / x["pick_us"] for x in r])),
                "within_5pct": float(np.mean([x["best_us"] / x["pick_us"] >= 1 / 1.05 for x in r])),
                "cold_start_speedup": sum(x["exhaustive_s"] for x in r) / sum(x["learned_s"] for x in r)}
            for k, r in by_k.items()}
    q = np.array([r["best_us"] / r["pick_us"] for r in rows])
    qd = np.array([r["best_us"] / r["default_us"] for r in rows])
    ls = sum(r["learned_s"] for r in rows)
    es = sum(r["exhaustive_s"] for r in rows)
    part = {}
    for name, sel in (("gemm_fp32", lambda r: not r["gemv"] and r["precision"] == L.GEMM_FP32),
                      ("gemm_bf16", lambda r: not r["gemv"] and r["precision"] == L.GEMM_BF16),
                      ("gemv_f32", lambda r: r["gemv"])):
        idx = [i for i, r in enumerate(rows) if sel(r)]
        part[name] = {"keys": len(idx), "pick_vs_best_geomean": gm(q[idx]),
                      "default_vs_best_geomean": gm(qd[idx]),
                      "within_5pct": float(np.mean(q[idx] >= 1 / 1.05)) if idx else None,
                      "cold_start_speedup": (sum(rows[i]["exhaustive_s"] for i in idx) /
                                             max(1e-9, sum(rows[i]["learned_s"] for i in idx))) if idx else None}
    return {
        "metric": "tune time learned vs exhaustive", "unit": "x (cold-start speedup)", "value": es / ls,
        "ms_per_step": 1e3 * ls / len(rows), "dtype": "f32/bf16", "higher_is_better": True,
        "config": {"workload": "learned GEMM/GEMV tuner: %d train + %d held-out keys, M,N,K log-uniform "
                               "[64,16384], seed 13" % (n_train, len(rows)), "top_k": 3,
                   "search_space": {"gemm": T.GEMM_SPACE, "gemv": T.GEMV_SPACE}},
        "tuner": {"pick_vs_best_geomean": gm(q), "within_5pct": float(np.mean(q >= 1 / 1.05)),
                  "default_vs_best_geomean": gm(qd), "learned_s_total": ls, "exhaustive_s_total": es,
                  "train_samples": len(samples), "train_loss": loss, "train_s": train_s, "sweep_s": sweep_s,
                  "by_kind": part, "top_k": topk},
        "e2e": None, "roofline": None, "clocks": clk.summary(), "steps": len(rows), "gpu_launches": None,
    }


TUNER_DB = ROOT / "chai_b200" / "data" / "tuner.db"     # trained by --workload tuner --save-db


def run_tuner_eval(args, L, ctx, stream):
    """The learned tuner on held-out keys with the committed cost model
    (chai_b200/data/tuner.db + .mlp, trained by `--workload tuner --save-db`
    on the 2000 training keys): the first TUNER_EVAL_KEYS of the 200 held-out
    keys (seed 13) are swept exhaustively, then tuned from cold by the learned
    method (rank every configuration, time the top 3) and by the exhaustive
    one; quality is judged on each key's own sweep (per-configuration median
    of 3 sweeps)."""
    import torch
    from chai_b200 import tuner as T
    import chai_b200.api as ch
    if not (TUNER_DB.exists() and TUNER_DB.with_name(TUNER_DB.name + ".mlp").exists()):
        raise RuntimeError("no trained cost model committed at chai_b200/data/tuner.db")
    n_eval = getattr(args, "tuner_eval_keys", 0) or TUNER_EVAL_KEYS
    held_keys = T.shapes(2200, seed=13)[2000:2000 + n_eval]
    held, _ = T.collect(ctx, held_keys, repeats=3)
    with Clocks(torch.cuda.current_device()) as clk:
        dev = ch.Device(config="TuneDB=%s TopK=3" % TUNER_DB)
        try:
            rows = T.evaluate(dev.ctx, held)
        finally:
            dev.close()
    gm = lambda v: float(np.exp(np.mean(np.log(v)))) if len(v) else None
    q = np.array([r["best_us"] / r["pick_us"] for r in rows])
    qd = np.array([r["best_us"] / r["default_us"] for r in rows])
    ls = sum(r["learned_s"] for r in rows)
    es = sum(r["exhaustive_s"] for r in rows)
    return {
        "metric": "tune time learned vs exhaustive", "unit": "x (cold-start speedup)", "value": es / ls,
        "ms_per_step": 1e3 * ls / len(rows), "steps": len(rows), "dtype": "f32/bf16", "higher_is_better": True,
        "config": {"workload": "learned GEMM/GEMV tuner, committed cost model, %d of the 200 held-out keys "
                               "(M,N,K log-uniform [64,16384], seed 13), top 3 timed" % len(rows)},
        "tuner": {"pick_vs_best_geomean": gm(q), "within_5pct": float(np.mean(q >= 1 / 1.05)),
                  "default_vs_best_geomean": gm(qd), "learned_s_total": ls, "exhaustive_s_total": es},
        "e2e": None, "roofline": None, "clocks": clk.summary(), "gpu_launches": None,
    }


TUNER_EVAL_KEYS = 40


WORKLOADS = {"gemm": run_gemm, "mc": run_mc, "mc-hbm": run_mc_hbm, "kirsch": run_kirsch, "gemv": run_gemv,
             "mc-many": run_mc_many, "grouped": run_grouped, "tuner": run_tuner, "c1": run_c1,
             "tuner-eval": run_tuner_eval}


# ---------------------------------------------------------------- reference arm

def workload_desc(args):
    """The workload names the two arms share (the same strings the GPU arm's
    `config.workload` carries)."""
    wl = args.workload
    if wl == "gemm":
        n = args.size or 16384
        return ("square GEMM M=N=K=%d, f32 operands uniform[-1,1) (chai Philox seeds 1,2), %s"
                % (n, args.precision)), args.precision
    if wl == "mc":
        return "Monte Carlo trace, 2^27 Philox4x32-10 Box-Muller normals, fused", "f32"
    if wl == "c1":
        return ("C1: A, B = chai Philox uniform[-1,1) 512x512 (seed 0), C = matmul(A, B), s = sum(C*C), one traced "
                "evaluation (plan replay)"), "f32"
    if wl == "mc-hbm":
        return "Monte Carlo payoff over 2^27 f32 normals already in HBM (materialised Z), fused", "f32"
    if wl == "kirsch":
        W = args.size or 8192
        return "Kirsch 8-direction compass filter via gather2_floor, %dx%d f32 uniform[0,1)" % (W, W), "f32"
    if wl == "gemv":
        m = args.size or 8192
        p = "f64" if args.precision == "f64" else "f32"
        return "GEMV y = A x, %dx%d %s" % (m, m, p), p
    if wl == "mc-many":
        return ("64 MC traces, lengths log-uniform in [2^12, 2^22] (seed 7), one persistent kernel + combine "
                "captured in a CUDA graph"), "f32"
    if wl == "grouped":
        return ("4096 grouped f32 GEMMs, M,N,K multiples of 8 in [32,512] (seed 11), one persistent tcgen05 "
                "launch"), "bf16x3"
    return wl, "f32"


def run_reference(args, steps=None):
    """The reference's own CPU implementation of the path -- its bytecode
    interpreter (runtime/Interpreter.cpp), built from the reference sources into
    oracle/_ref -- timed on this host on a bounded sample of the same workload.
    The interpreter is one device thread (runtime/DeviceMap.cpp:17-23), so it
    uses one core whatever the host offers."""
    drv = ROOT / "oracle" / "_ref" / "ref_driver"
    if not drv.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_driver not built (reference sources absent)"}
    steps = steps or max(1, args.steps)
    wl = args.workload
    if wl in ("tuner", "tuner-eval"):
        return {"impl": "reference", "unavailable": "the reference tuner (StandardEM over generated OpenCL "
                                                   "kernels) needs an OpenCL GPU device; none on this host"}
    times = []
    with tempfile.TemporaryDirectory() as td:
        rng = np.random.default_rng(1)
        if wl == "gemm":
            n = 512      # the reference's own CPU-runnable matmul size; 1024^3 takes ~18 s per run
            rng.uniform(-1, 1, (n, n)).astype(np.float32).tofile(td + "/A")
            rng.uniform(-1, 1, (n, n)).astype(np.float32).tofile(td + "/B")
            cmd = [str(drv), "gemm_f32", str(n), str(n), str(n), td + "/A", td + "/B", td + "/C"]
            unit, metric = "TFLOP/s", "GEMM TFLOP/s at err vs FP32"
            conv = lambda ms: 2.0 * n ** 3 / (ms * 1e-3) / 1e12
            sample = "interpreter matmul 512^3 f32 (f32 products summed in double), inputs via make2"
        elif wl == "c1":
            n = C1_N
            rng.uniform(-1, 1, (n, n)).astype(np.float32).tofile(td + "/A")
            rng.uniform(-1, 1, (n, n)).astype(np.float32).tofile(td + "/B")
            cmd = [str(drv), "matmul_sum", str(n), td + "/A", td + "/B", td + "/C", td + "/s"]
            unit, metric = "TFLOP/s", "C1 trace TFLOP/s (512^3 matmul + sum(C*C))"
            conv = lambda ms: (2.0 * n ** 3 + 2.0 * n * n) / (ms * 1e-3) / 1e12
            sample = "the whole C1 trace in the interpreter (make2 inputs, matmul 512^3, sum(C*C), read-back)"
        elif wl == "grouped":
            cmd = None
            unit, metric = "TFLOP/s", "GEMM TFLOP/s at err vs FP32"
            sample = "interpreter matmul loop over the first 16 of the 4096 grouped problems"
            shapes = grouped_shapes()[:16]
            files = []
            for i, (m, n, k) in enumerate(shapes):
                rng.uniform(-1, 1, (m, k)).astype(np.float32).tofile(td + "/A%d" % i)
                rng.uniform(-1, 1, (k, n)).astype(np.float32).tofile(td + "/B%d" % i)
        elif wl == "mc-many":
            Ls = [max(4, L // 16) for L in many_lengths()]
            cmd = None
            unit, metric = "Gnormals/s", "trace throughput (64 uneven MC traces, one persistent launch)"
            sample = "64 sequential interpreter MC traces, lengths 1/16 of the GPU workload's"
        elif wl == "mc-hbm":
            n = 1 << 19
            rng.standard_normal(n).astype(np.float32).tofile(td + "/Z")
            cmd = [str(drv), "mc", str(n), td + "/Z"]
            unit, metric = "GB/s", "trace HBM GB/s"
            conv = lambda ms: 4 * n / (ms * 1e-3) / 1e9
            sample = "interpreter MC payoff over 2^19 given normals (make1)"
        elif wl == "mc":
            W, H = 1024, 512
            cmd = [str(drv), "mc_rng", str(W), str(H)]
            unit, metric = "Gnormals/s", "trace throughput (MC: Philox normals -> exp -> mean)"
            conv = lambda ms: W * H / (ms * 1e-3) / 1e9
            sample = "interpreter MC trace over 2^19 normals (its own RNG)"
        elif wl == "kirsch":
            W = H = 1024
            rng.uniform(0, 1, (H, W)).astype(np.float32).tofile(td + "/img")
            cmd = [str(drv), "kirsch", str(W), str(H), td + "/img", td + "/out"]
            unit, metric = "GB/s", "trace HBM GB/s"
            conv = lambda ms: 2 * 4 * W * H / (ms * 1e-3) / 1e9
            sample = "interpreter Kirsch trace (8 gather2_floor + max) over 1024x1024"
        else:
            m = n = 4096
            rng.uniform(-1, 1, (m, n)).astype(np.float32).tofile(td + "/A")
            rng.uniform(-1, 1, n).astype(np.float32).tofile(td + "/x")
            cmd = [str(drv), "gemv_f32", str(m), str(n), td + "/A", td + "/x", td + "/y"]
            unit, metric = "GB/s", "GEMV GB/s"
            conv = lambda ms: (m * n + m + n) * 4 / (ms * 1e-3) / 1e9
            sample = "interpreter matmul(matrix, vector) 4096x4096 f32"
        for _ in range(steps):
            if wl == "grouped":     # one interpreter matmul per problem
                ms_sum = 0.0
                for i, (m, n, k) in enumerate(shapes):
                    r = subprocess.run([str(drv), "gemm_f32", str(m), str(n), str(k), td + "/A%d" % i, td + "/B%d" % i,
                                        td + "/C"], capture_output=True, text=True, timeout=600)
                    if r.returncode != 0:
                        return {"impl": "reference", "unavailable": "ref_driver failed: " + r.stderr[-200:]}
                    ms_sum += float(r.stdout.split("ms=")[1].split()[0])
                times.append(ms_sum)
                conv = lambda ms: sum(2.0 * m * n * k for m, n, k in shapes) / (ms * 1e-3) / 1e12
                continue
            if wl == "mc-many":     # the reference runs uneven traces one dispatch at a time
                ms_sum = 0.0
                for L in Ls:
                    r = subprocess.run([str(drv), "mc_rng", str(L), "1"], capture_output=True, text=True, timeout=600)
                    if r.returncode != 0:
                        return {"impl": "reference", "unavailable": "ref_driver failed: " + r.stderr[-200:]}
                    ms_sum += float(r.stdout.split("ms=")[1].split()[0])
                times.append(ms_sum)
                conv = lambda ms: sum(Ls) / (ms * 1e-3) / 1e9
                continue
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                return {"impl": "reference", "unavailable": "ref_driver failed: " + r.stderr[-200:]}
            times.append(float(r.stdout.split("ms=")[1].split()[0]))
    ms = statistics.median(times)
    v = conv(ms)
    desc, _ = workload_desc(args)
    return {"impl": "reference", "metric": metric, "value": v, "unit": unit, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if (wl == "gemv" and args.precision == "f64") else "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": desc, "reference_sample": sample,
                       "parallelism": "one interpreter device thread (runtime/DeviceMap.cpp:17-23)"},
            "cpu_baseline": {"value": v, "unit": unit, "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline(args):
    r = run_reference(args, steps=2)
    return r.get("cpu_baseline") if "cpu_baseline" in r else {"unavailable": r.get("unavailable")}


# ---------------------------------------------------------------- main

# The other parts of the benchmark metric, measured in the default run after
# the headline GEMM: trace HBM GB/s (materialised MC, Kirsch), the fused MC
# trace (issue-bound), the 64 uneven traces, the grouped GEMM, GEMV f32 / f64,
# the C1 trace and the learned tuner's held-out evaluation.  Each timed region
# lasts at least SECONDARY_MIN_S seconds so the clock sampler records it.
SECONDARY = [("mc_hbm", "mc-hbm", {}), ("kirsch", "kirsch", {}), ("mc", "mc", {}), ("mc_many", "mc-many", {}),
             ("grouped", "grouped", {"precision": "bf16x3"}), ("gemv_f32", "gemv", {"precision": "f32"}),
             ("gemv_f64", "gemv", {"precision": "f64"}), ("c1", "c1", {}), ("tuner", "tuner-eval", {})]
SECONDARY_MIN_S = 1.2


def secondary(args, L, ctx, stream):
    import torch
    out = {}
    for key, wl, over in SECONDARY:
        a = argparse.Namespace(**vars(args))
        a.workload, a.size, a.precision, a.min_timed_s = wl, 0, "bf16x3", SECONDARY_MIN_S
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        try:
            r = WORKLOADS[wl](a, L, ctx, stream)
        except Exception as e:          # one failed part must not hide the others
            out[key] = {"error": "%s: %s" % (type(e).__name__, str(e)[:300])}
            continue
        finally:
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        item = {k: r.get(k) for k in ("metric", "value", "unit", "ms_per_step", "steps", "dtype", "e2e", "roofline",
                                     "clocks", "gpu_launches", "tuner") if r.get(k) is not None}
        item["config"] = r.get("config")
        if not args.no_cpu_baseline and wl != "tuner-eval":
            item["cpu_baseline"] = cpu_baseline(a)
        item["wall_s"] = time.perf_counter() - t0
        out[key] = item
    return out


def aggregate_ranks(res, world, reduce_max):
    """Whole-job figures from one rank's result under weak scaling: every rank
    processes the same per-GPU workload, the job's step time is the maximum
    over ranks (reduce_max: the collective), and `value` becomes the units all
    ranks processed divided by that time.  The end-to-end figure is
    aggregated the same way from the slowest rank's end-to-end rate."""
    local_ms = res["ms_per_step"]
    ms = reduce_max(local_ms)
    res["value"] = res["value"] * world * local_ms / ms
    res["ms_per_step"] = ms
    # every rank takes part in the collective, with or without an e2e figure
    e2e = res.get("e2e")
    v = e2e["value"] if e2e and e2e.get("value") else float("inf")
    slowest = -reduce_max(-v)                      # min over ranks (higher is better)
    if e2e and math.isfinite(slowest):
        res["e2e"] = dict(e2e, value=slowest * world, per_rank_min=slowest)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="gemm", choices=sorted(WORKLOADS))
    ap.add_argument("--sweep", default="", help="gemm only: write the precision/error sweep JSON here")
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--size", type=int, default=0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--save-db", action="store_true",
                    help="tuner: write the trained cost model to chai_b200/data/tuner.db")
    ap.add_argument("--no-secondary", action="store_true",
                    help="default run: skip the secondary measurements after the headline GEMM")
    ap.add_argument("--config", default=None, help="back-end configuration string (chai_cuda_init)")
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
    os.environ.setdefault("CHAI_KERNEL_TIMING", "1")
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
    dev = ch.init(config=args.config, device=local)
    stream = torch.cuda.Stream()          # one stream shared by torch events and the library
    torch.cuda.set_stream(stream)
    L.lib().chai_cuda_set_stream(dev.ctx, C.c_void_p(stream.cuda_stream))
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    res = WORKLOADS[args.workload](args, L, dev.ctx, stream)
    if args.sweep and args.workload == "gemm":
        gemm_sweep(args, L, dev.ctx, stream, args.sweep)
    torch.cuda.synchronize()
    if pg:
        def reduce_max(x):
            t = torch.tensor([x], device="cuda", dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            return float(t.item())
        aggregate_ranks(res, world, reduce_max)
    if rank == 0:
        line = {"metric": res["metric"], "value": res["value"], "unit": res["unit"], "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": res["higher_is_better"], "scaling": "weak", "vs_baseline": None,
                "dtype": res["dtype"], "data": "synthetic (seeded)",
                "config": dict(res["config"], parallelism="independent traces per GPU (dp%d)" % world)}
        for k in ("e2e", "roofline", "clocks", "gpu_launches"):
            line[k] = res.get(k)
        if "tuner" in res:
            line["tuner"] = res["tuner"]
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args)
        if world == 1 and args.workload == "gemm" and not args.no_secondary and not args.sweep:
            line["secondary"] = secondary(args, L, dev.ctx, stream)
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    ch.shutdown()


if __name__ == "__main__":
    main()
