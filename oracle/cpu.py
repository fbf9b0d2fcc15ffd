"""ctypes access to the oracle's C restatement (oracle/_build/liboracle.so).

Test infrastructure only (see oracle/__init__.py)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None

PHILOX, THREEFRY = 1230, 1231
U32, I32, F32, F64 = 0, 1, 4, 8
LAYOUT_CHAI, LAYOUT_COUNTER = 0, 1
JIT_PI = 3.14159  # M_PI as the reference JIT prints it (6 significant digits)

__all__ = ["lib", "rng_fill", "gemm_f64", "matmul_ref", "matvec_ref", "gemm_entries_f64", "gemv_f64", "sum_f32", "dot_f32",
           "gather2_floor", "kirsch", "philox4x32", "philox2x32", "philox2x64", "threefry4x32",
           "threefry4x32_chai", "threefry2x32", "threefry2x64", "PHILOX", "THREEFRY", "U32", "I32",
           "F32", "F64", "LAYOUT_CHAI", "LAYOUT_COUNTER", "JIT_PI"]


def lib():
    global _LIB
    if _LIB is None:
        so = HERE / "_build" / "liboracle.so"
        if not so.exists():
            from . import build_ref
            build_ref.build_oracle()
        _LIB = C.CDLL(str(so))
        L = _LIB
        p = C.c_void_p
        L.chai_rng_fill.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                    C.c_size_t, C.c_int, C.c_double, C.c_double, C.c_double, p]
        L.oracle_gemm_f32_to_f64.argtypes = [C.c_int64] * 3 + [p] * 3
        L.oracle_gemm_entries_f64.argtypes = [C.c_int64, C.c_int64, p, p, C.c_int64, p, p, p]
        L.oracle_gemv_f64.argtypes = [C.c_int64, C.c_int64, p, p, p]
        L.oracle_gemv_f32.argtypes = [C.c_int64, C.c_int64, p, p, p]
        L.oracle_matmul_ref_f32.argtypes = [C.c_int64] * 4 + [p] * 3
        L.oracle_matvec_ref_f32.argtypes = [C.c_int64] * 3 + [p] * 3
        L.oracle_sum_f32.argtypes = [C.c_int64, p]
        L.oracle_sum_f32.restype = C.c_double
        L.oracle_dot_f32.argtypes = [C.c_int64, p, p]
        L.oracle_dot_f32.restype = C.c_double
        L.oracle_gather2_floor_f32.argtypes = [C.c_int64, C.c_int64, p, p, p, p]
        L.oracle_kirsch_f32.argtypes = [C.c_int64, C.c_int64, p, p]
        for n in ("r123_philox2x32", "r123_philox4x32", "r123_philox2x64", "r123_threefry2x32",
                  "r123_threefry4x32", "r123_threefry4x32_chai", "r123_threefry2x64"):
            getattr(L, n).argtypes = [p, p, p]
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def rng_fill(n: int, *, variant=PHILOX, prec=F32, vec_len=None, dist=0, layout=LAYOUT_CHAI, seed=0,
             first_vec=0, limits=None, pi=JIT_PI) -> np.ndarray:
    """Chai array of n random elements (see r123.h for the layout)."""
    if vec_len is None:
        vec_len = 2 if prec == F64 else 4
    dt = {U32: np.uint32, I32: np.int32, F32: np.float32, F64: np.float64}[prec]
    out = np.empty(n, dtype=dt)
    lo, hi = (limits if limits is not None else (0.0, 1.0))
    lib().chai_rng_fill(variant, prec, vec_len, dist, layout, seed, first_vec, n,
                        1 if limits is not None else 0, float(lo), float(hi), pi, _ptr(out))
    return out


def gemm_f64(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, K = A.shape
    K2, N = B.shape
    assert K == K2
    Cm = np.empty((M, N), dtype=np.float64)
    lib().oracle_gemm_f32_to_f64(M, N, K, _ptr(A), _ptr(B), _ptr(Cm))
    return Cm


def matmul_ref(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """The reference interpreter's f32 matmul: f32 products accumulated in
    double, k ascending (interp/InterpMatmulBase.hpp:50-61)."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, Ka = A.shape
    Kb, N = B.shape
    out = np.empty((M, N), dtype=np.float32)
    lib().oracle_matmul_ref_f32(M, N, Ka, Kb, _ptr(A), _ptr(B), _ptr(out))
    return out


def matvec_ref(A: np.ndarray, x: np.ndarray) -> np.ndarray:
    """The interpreter's f32 matrix-vector product (InterpMatmulBase.hpp:37-47)."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(A.shape[0], dtype=np.float32)
    lib().oracle_matvec_ref_f32(A.shape[0], A.shape[1], x.shape[0], _ptr(A), _ptr(x), _ptr(out))
    return out


def gemm_entries_f64(A, B, rows, cols) -> np.ndarray:
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    out = np.empty(rows.shape[0], dtype=np.float64)
    lib().oracle_gemm_entries_f64(B.shape[1], A.shape[1], _ptr(A), _ptr(B), rows.shape[0], _ptr(rows),
                                  _ptr(cols), _ptr(out))
    return out


def gemv_f64(A: np.ndarray, x: np.ndarray) -> np.ndarray:
    M, N = A.shape
    y = np.empty(M, dtype=np.float64)
    if A.dtype == np.float64:
        A = np.ascontiguousarray(A)
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().oracle_gemv_f64(M, N, _ptr(A), _ptr(x), _ptr(y))
    else:
        A = np.ascontiguousarray(A, dtype=np.float32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        lib().oracle_gemv_f32(M, N, _ptr(A), _ptr(x), _ptr(y))
    return y


def sum_f32(a: np.ndarray) -> float:
    a = np.ascontiguousarray(a, dtype=np.float32).ravel()
    return lib().oracle_sum_f32(a.size, _ptr(a))


def dot_f32(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, dtype=np.float32).ravel()
    b = np.ascontiguousarray(b, dtype=np.float32).ravel()
    return lib().oracle_dot_f32(a.size, _ptr(a), _ptr(b))


def gather2_floor(A: np.ndarray, X: np.ndarray, Y: np.ndarray) -> np.ndarray:
    H, W = A.shape
    A = np.ascontiguousarray(A, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    out = np.empty_like(A)
    lib().oracle_gather2_floor_f32(W, H, _ptr(A), _ptr(X), _ptr(Y), _ptr(out))
    return out


def kirsch(A: np.ndarray) -> np.ndarray:
    H, W = A.shape
    A = np.ascontiguousarray(A, dtype=np.float32)
    out = np.empty_like(A)
    lib().oracle_kirsch_f32(W, H, _ptr(A), _ptr(out))
    return out


def _bij(name, width, ctr, key, nout):
    dt = np.uint64 if width == 64 else np.uint32
    c = np.ascontiguousarray(ctr, dtype=dt)
    k = np.ascontiguousarray(key, dtype=dt)
    o = np.empty(nout, dtype=dt)
    getattr(lib(), name)(_ptr(c), _ptr(k), _ptr(o))
    return o


def philox4x32(ctr, key): return _bij("r123_philox4x32", 32, ctr, key, 4)
def philox2x32(ctr, key): return _bij("r123_philox2x32", 32, ctr, key, 2)
def philox2x64(ctr, key): return _bij("r123_philox2x64", 64, ctr, key, 2)
def threefry4x32(ctr, key): return _bij("r123_threefry4x32", 32, ctr, key, 4)
def threefry4x32_chai(ctr, key): return _bij("r123_threefry4x32_chai", 32, ctr, key, 4)
def threefry2x32(ctr, key): return _bij("r123_threefry2x32", 32, ctr, key, 2)
def threefry2x64(ctr, key): return _bij("r123_threefry2x64", 64, ctr, key, 2)
