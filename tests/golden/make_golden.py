"""Generate the golden fixtures in this directory from the reference itself.

Run with the reference checkout named (the oracle recipe oracle/build_ref.py
compiles its sources into oracle/_ref/):

    python tests/golden/make_golden.py --reference <reference checkout>

(or CHAI_REFERENCE=<reference checkout> in the environment).

Fixtures (numpy .npz, a few hundred KB in all):
  r123_bijections.npz  Philox2x32/4x32/2x64 and Threefry2x32/4x32/2x64 outputs
                       on seeded counters and keys, from the Random123 text the
                       reference JIT prints (Random123/R123Philox.cpp,
                       Random123/R123Threefry.cpp; libr123_jit.so) and from the
                       vendored upstream Random123 text (Random123/r123*.i;
                       libr123_upstream.so)
  r123_wrappers.npz    every per-variant uniform / normal wrapper of the JIT
                       text (chai's key / counter layout and its int -> float
                       conversions) at seeded and edge (tid, idx) pairs
                       (libr123_wrappers.so)
  interp.npz           traces run on the reference's bytecode interpreter
                       (oracle/_ref/ref_driver): matmul + sum at 512 x 512 (the
                       small plain-matmul workload), ragged f32 / f64 matmul,
                       f32 / f64 matrix-vector, the Kirsch gather2_floor stencil,
                       sum / mean / dot_product and the Monte Carlo payoff

Inputs come from numpy's seeded generator except the 512 x 512 matmul, whose
inputs are Philox4x32-10 uniforms in [-1, 1) with counter = element index / 4
and key 0 for A, key 1 for B (the oracle's counter layout, itself pinned by the
bijection fixtures).
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import build_ref  # noqa: E402

REF = ROOT / "oracle" / "_ref"
GENS = {"philox2x32": (32, 2, 1), "philox4x32": (32, 4, 2), "philox2x64": (64, 2, 1),
        "threefry2x32": (32, 2, 2), "threefry4x32": (32, 4, 4), "threefry2x64": (64, 2, 2)}


def _bijections(rng):
    jit = C.CDLL(str(REF / "libr123_jit.so"))
    up = C.CDLL(str(REF / "libr123_upstream.so"))
    out = {}
    for name, (bits, nc, nk) in GENS.items():
        dt = np.uint32 if bits == 32 else np.uint64
        ctr = rng.integers(0, 2 ** bits, (64, nc), dtype=dt)
        key = rng.integers(0, 2 ** bits, (64, nk), dtype=dt)
        ctr[0] = 0
        key[0] = 0
        ctr[1] = np.iinfo(dt).max
        key[1] = np.iinfo(dt).max
        for tag, lib in (("jit", jit), ("up", up)):
            f = getattr(lib, "%s_%s" % (tag, name))
            f.argtypes = [C.c_void_p] * 3
            res = np.zeros((64, nc), dtype=dt)
            for i in range(64):
                c, k = np.ascontiguousarray(ctr[i]), np.ascontiguousarray(key[i])
                f(c.ctypes.data, k.ctypes.data, res[i].ctypes.data)
            out["%s_%s" % (name, tag)] = res
        out[name + "_ctr"] = ctr
        out[name + "_key"] = key
    return out


def _wrappers(rng):
    so = build_ref.build_r123_wrapper_pins()
    lib = C.CDLL(str(so))
    text = (REF / "r123_jit.cl").read_text()
    import re
    sigs = re.findall(r"^inline (\w+) ((?:philox|threefry)_(?:uniform|normal)_(\d+)_(\d+))\(", text, flags=re.M)
    tid = np.concatenate([[0, 1, 2, 3, 2 ** 31 - 1, 2 ** 31, 2 ** 32 - 1], rng.integers(0, 2 ** 32, 41)]).astype(np.uint64)
    idx = np.concatenate([[0, 0, 42, 7, 1, 2 ** 32 - 1, 0], rng.integers(0, 2 ** 32, 41)]).astype(np.uint64)
    out = {"tid": tid, "idx": idx}
    seen = set()
    for rt, name, prec, lanes in sigs:
        if name in seen:
            continue
        seen.add(name)
        prec, lanes = int(prec), int(lanes)
        dt = {0: np.uint32, 1: np.int32, 4: np.float32, 8: np.float64}[prec]
        f = getattr(lib, "w_" + name)
        f.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p]
        res = np.zeros((tid.size, lanes), dtype=dt)
        for i in range(tid.size):
            f(int(tid[i]), int(idx[i]), res[i].ctypes.data)
        out[name] = res
    return out


def _drv(*args):
    r = subprocess.run([str(REF / "ref_driver"), *map(str, args)], capture_output=True, text=True, check=True)
    return dict(kv.split("=") for kv in r.stdout.split())


def _interp(rng):
    import oracle
    out = {}
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)

        def put(name, a):
            a.tofile(t / name)
            return t / name

        # the small plain-matmul trace: C = matmul(A, B), s = sum(C * C), 512 x 512
        n = 512
        A = oracle.rng_fill(n * n, layout=oracle.LAYOUT_COUNTER, seed=0, limits=(-1.0, 1.0)).reshape(n, n)
        B = oracle.rng_fill(n * n, layout=oracle.LAYOUT_COUNTER, seed=1, limits=(-1.0, 1.0)).reshape(n, n)
        kv = _drv("matmul_sum", n, put("A", A), put("B", B), t / "C", t / "s")
        Cm = np.fromfile(t / "C", dtype=np.float32).reshape(n, n)
        out["mm512_s"] = np.float32(float(kv["s"]))
        out["mm512_rowsum"] = Cm.astype(np.float64).sum(axis=1)
        sel = rng.integers(0, n, (256, 2))
        out["mm512_sel"] = sel
        out["mm512_C_sel"] = Cm[sel[:, 0], sel[:, 1]]
        out["mm512_A_head"] = A[:2].copy()
        out["mm512_B_head"] = B[:2].copy()
        # ragged GEMM f32 / f64
        for tag, dt, (M, N, K) in (("f32", np.float32, (37, 53, 29)), ("f64", np.float64, (19, 23, 31))):
            A = rng.uniform(-1, 1, (M, K)).astype(dt)
            B = rng.uniform(-1, 1, (K, N)).astype(dt)
            _drv("gemm_" + tag, M, N, K, put("A", A), put("B", B), t / "C")
            out["gemm_%s_A" % tag], out["gemm_%s_B" % tag] = A, B
            out["gemm_%s_C" % tag] = np.fromfile(t / "C", dtype=dt).reshape(M, N)
        # matrix-vector f32 / f64
        for tag, dt in (("f32", np.float32), ("f64", np.float64)):
            M, N = 61, 47
            A = rng.uniform(-1, 1, (M, N)).astype(dt)
            x = rng.uniform(-1, 1, N).astype(dt)
            _drv("gemv_" + tag, M, N, put("A", A), put("x", x), t / "y")
            out["gemv_%s_A" % tag], out["gemv_%s_x" % tag] = A, x
            out["gemv_%s_y" % tag] = np.fromfile(t / "y", dtype=dt)
        # Kirsch stencil through gather2_floor (periodic wrap), ragged 40 x 24
        W, H = 40, 24
        img = rng.uniform(0, 1, (H, W)).astype(np.float32)
        _drv("kirsch", W, H, put("img", img), t / "k")
        out["kirsch_img"] = img
        out["kirsch_out"] = np.fromfile(t / "k", dtype=np.float32).reshape(H, W)
        # reductions
        W, H = 100, 7
        a = rng.uniform(-1, 1, (H, W)).astype(np.float32)
        b = rng.uniform(-1, 1, (H, W)).astype(np.float32)
        kv = _drv("reduce", W, H, put("a", a), put("b", b))
        out["reduce_a"], out["reduce_b"] = a, b
        out["reduce_sum_mean_dot"] = np.array([float(kv["sum"]), float(kv["mean"]), float(kv["dot"])],
                                              dtype=np.float32)
        # Monte Carlo payoff on given normals
        Z = rng.standard_normal(4096).astype(np.float32)
        kv = _drv("mc", Z.size, put("Z", Z))
        out["mc_Z"] = Z
        out["mc_payoff"] = np.float32(float(kv["payoff"]))
    return out


def main():
    if "--reference" in sys.argv:
        build_ref.set_reference(sys.argv[sys.argv.index("--reference") + 1])
    if not build_ref.available():
        raise SystemExit("name the reference checkout: --reference PATH or CHAI_REFERENCE")
    build_ref.build_all()
    rng = np.random.default_rng(20240613)
    np.savez_compressed(HERE / "r123_bijections.npz", **_bijections(rng))
    np.savez_compressed(HERE / "r123_wrappers.npz", **_wrappers(rng))
    np.savez_compressed(HERE / "interp.npz", **_interp(rng))
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
