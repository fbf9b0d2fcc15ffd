"""Running the reference's sample programs, unchanged, through the reference's
own front end linked with chai_b200 (oracle/build_ref.py build_cuda_frontend:
oracle/_ref/cuda/<sample>).  Shared by the CPU test (interpreter device, the
adapter's DeviceMap without CHAI_CUDA) and the GPU test (CudaDevice).

Expected outputs:
  - samples the interpreter runs: the same binary on the interpreter device
    (runtime/Interpreter.cpp), numbers compared with a relative tolerance;
  - samples with inline OpenCL (the interpreter has none,
    runtime/Interpreter.cpp:159-162): the sample's arithmetic restated here.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
SAMPLE_DIR = ROOT / "oracle" / "_ref" / "cuda"

# samples the interpreter device runs (compared against it)
INTERP_SAMPLES = ["matmul_uni", "matmul_vec", "matmul_pth", "matmul64_uni", "sum_uni", "sum_vec", "sum_pth",
                  "loopsum_uni", "loopsum_vec", "cg", "cg64", "index", "md5", "mingle", "filter", "kirch",
                  "american_option"]
# samples with inline OpenCL kernels (compared against restatements)
CL_SAMPLES = ["inline_cl", "bitonic", "american_option_batch"]

NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")


def available() -> bool:
    return (SAMPLE_DIR / "libchai_ref_cuda.so").exists() and all(
        (SAMPLE_DIR / s).exists() for s in INTERP_SAMPLES + CL_SAMPLES + ["pi"])


def run(sample: str, cuda: bool, timeout: int = 60) -> str:
    spec = SAMPLE_DIR / "interp.spec"
    if not spec.exists():
        spec.write_text("EnableInterpreter\n")
    env = dict(os.environ)
    env.pop("CHAI_CUDA", None)
    if cuda:
        env["CHAI_CUDA"] = "1"
    r = subprocess.run([str(SAMPLE_DIR / sample), "-f", str(spec)], capture_output=True, text=True, env=env,
                       timeout=timeout, cwd=str(SAMPLE_DIR))
    assert r.returncode == 0, (sample, cuda, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def same_output(a: str, b: str, rel: float = 1e-4, abs_: float = 1e-4) -> bool:
    """Same text with numbers equal within `rel` (relative) or `abs_`; hex
    digests and other words must match exactly."""
    if NUM.sub("#", a) != NUM.sub("#", b):
        return False
    for x, y in zip(NUM.findall(a), NUM.findall(b)):
        fx, fy = float(x), float(y)
        if not (fx == fy or abs(fx - fy) <= max(rel * max(abs(fx), abs(fy)), abs_)):
            return False
    return True


# ---- restatements of the inline-OpenCL samples

def expect_inline_cl() -> list[float]:
    """sample/inline_cl.cpp: C = A + B; C[i] += 1.5 (kernel); C += A - 3.3
    with A[i] = i, B[i] = 20 - i, in f32."""
    import numpy as np
    f = np.float32
    A = np.arange(20, dtype=f)
    B = f(20) - A
    C = (A + B) + f(1.5)
    C = C + (A - f(3.3))
    return [float(v) for v in C]


def glibc_random(n: int) -> list[int]:
    """The sample's random() stream (glibc, default seed 1)."""
    libc = C.CDLL("libc.so.6")
    libc.random.restype = C.c_long
    libc.srandom(1)
    return [int(libc.random()) & 0xFFFFFFFF for _ in range(n)]


def expect_american_batch() -> list[float]:
    """sample/finance/american_option_batch.cpp: 20 binomial trees (100 steps)
    over a volatility smile, in double, in the kernel's order of operations."""
    price, rate, maturity, steps, num = 100.0, 0.10, 1.0, 100, 20
    out = []
    for i in range(num):
        X = 100.0 - num // 2 + i
        vol = 0.25 + 0.1 * 4 * (i - num // 2) * (i - num // 2) / (num * num)
        R = math.exp(rate * (maturity / steps))
        up = math.exp(vol * math.sqrt(maturity / steps))
        down = 1.0 / up
        pr = (R - down) / (up - down)
        tmp = price * math.pow(down, steps)
        prices = [0.0] * (steps + 1)
        option = [0.0] * (steps + 1)
        prices[0], option[0] = tmp, max(tmp - X, 0.0)
        for k in range(1, steps + 1):
            tmp = tmp * up * up
            prices[k], option[k] = tmp, max(tmp - X, 0.0)
        for k in range(steps, 0, -1):
            for j in range(k):
                tmp = (pr * option[j + 1] + (1.0 - pr) * option[j]) / R
                prices[j] = down * prices[j + 1]
                option[j] = max(prices[j] - X, tmp)
        out.append(option[0])
    return out
