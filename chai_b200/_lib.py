"""ctypes binding of the C ABI declared in include/chai_b200.h.

The shared library is built in-tree (chai_b200/libchai_b200.so, see build.py).
There is no CPU fallback: if the library is missing, loading fails loudly, and
every compute entry point needs an sm_100 GPU (CHAI_ERR_NO_DEVICE otherwise).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libchai_b200.so"

CHAI_OK = 0
ERR = {-1: "INVALID", -2: "UNSUPPORTED", -3: "OOM", -4: "LAUNCH", -5: "TIMEOUT", -6: "NOT_FOUND",
       -7: "NO_DEVICE", -8: "JIT", -9: "INJECTED"}
U32, I32, F32, F64 = 0, 1, 4, 8
PHILOX, THREEFRY = 1230, 1231
BC_OPCODE, BC_VARIABLE, BC_SCALAR, BC_MEMORY, BC_KERNEL = 0, 1, 2, 3, 4
KARG_ARRAY, KARG_LOCAL, KARG_SCALAR = 0, 1, 2
GEMM_FP32, GEMM_TF32, GEMM_BF16, GEMM_BF16X3, GEMM_BF16X6, GEMM_FP8, GEMM_FP64, GEMM_AUTO = range(8)
TUNE_LEARNED, TUNE_EXHAUSTIVE, TUNE_DEFAULT = 0, 1, 2


class chai_bc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("code", C.c_uint32), ("version", C.c_uint32), ("reserved", C.c_uint32),
                ("scalar", C.c_double), ("buffer", C.c_uint64)]


class chai_stmt(C.Structure):
    _fields_ = [("lhs_variable", C.c_uint32), ("lhs_version", C.c_uint32), ("n_cells", C.c_uint32),
                ("reserved", C.c_uint32), ("cells", C.POINTER(chai_bc))]


class chai_kernel_arg(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("prec", C.c_uint32), ("variable", C.c_uint32), ("version", C.c_uint32),
                ("value", C.c_double)]


class chai_inline_kernel(C.Structure):
    _fields_ = [("source", C.c_char_p), ("name", C.c_char_p), ("n_args", C.c_uint32), ("reserved", C.c_uint32),
                ("args", C.POINTER(chai_kernel_arg)), ("global_size", C.c_uint64 * 2),
                ("local_size", C.c_uint64 * 2)]


class chai_trace_desc(C.Structure):
    _fields_ = [("num_traces", C.c_uint32), ("n_stmts", C.c_uint32), ("stmts", C.POINTER(chai_stmt)),
                ("hash", C.c_uint64), ("kernels", C.POINTER(chai_inline_kernel)), ("n_kernels", C.c_uint32),
                ("reserved", C.c_uint32)]


class chai_buffer_binding(C.Structure):
    _fields_ = [("variable", C.c_uint32), ("prec", C.c_uint32), ("width", C.c_uint64), ("height", C.c_uint64),
                ("slots", C.c_uint32), ("reserved", C.c_uint32), ("buffer", C.c_uint64)]


class chai_value_shape(C.Structure):
    _fields_ = [("variable", C.c_uint32), ("version", C.c_uint32), ("prec", C.c_uint32), ("slots", C.c_uint32),
                ("width", C.c_uint64), ("height", C.c_uint64)]


class chai_rng_desc(C.Structure):
    _fields_ = [("variant", C.c_uint32), ("prec", C.c_uint32), ("dist", C.c_uint32), ("vec_len", C.c_uint32),
                ("seed", C.c_uint64), ("width", C.c_uint64), ("height", C.c_uint64), ("slots", C.c_uint32),
                ("has_limits", C.c_uint32), ("min_limit", C.c_double), ("max_limit", C.c_double)]


class chai_gemm_desc(C.Structure):
    _fields_ = [("precision", C.c_int32), ("trans_a", C.c_int32), ("trans_b", C.c_int32), ("reserved", C.c_int32),
                ("m", C.c_int64), ("n", C.c_int64), ("k", C.c_int64),
                ("a", C.c_void_p), ("lda", C.c_int64), ("b", C.c_void_p), ("ldb", C.c_int64),
                ("c", C.c_void_p), ("ldc", C.c_int64), ("alpha", C.c_double), ("beta", C.c_double),
                ("batch", C.c_int64), ("stride_a", C.c_int64), ("stride_b", C.c_int64), ("stride_c", C.c_int64)]


class chai_gemm_problem(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("k", C.c_int32), ("reserved", C.c_int32),
                ("a", C.c_void_p), ("b", C.c_void_p), ("c", C.c_void_p)]


class chai_gemm_key(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("k", C.c_int64), ("precision", C.c_int32),
                ("is_gemv", C.c_int32)]


class chai_gemm_cfg(C.Structure):
    _fields_ = [("block_m", C.c_int32), ("block_n", C.c_int32), ("block_k", C.c_int32), ("stages", C.c_int32),
                ("vec_width", C.c_int32), ("cluster_m", C.c_int32), ("cluster_n", C.c_int32),
                ("group_m", C.c_int32), ("measured_us", C.c_double)]


P = C.c_void_p
# name -> (restype, argtypes); every symbol include/chai_b200.h declares
SIGNATURES = {
    "chai_cuda_init": (C.c_int, [C.c_int, C.c_char_p, C.POINTER(P)]),
    "chai_cuda_shutdown": (C.c_int, [P]),
    "chai_cuda_synchronize": (C.c_int, [P]),
    "chai_cuda_selftest_wait": (C.c_int, [P, C.c_double]),
    "chai_cuda_error_string": (C.c_char_p, [C.c_int]),
    "chai_cuda_last_error": (C.c_char_p, [P]),
    "chai_cuda_set_stream": (C.c_int, [P, P]),
    "chai_cuda_kernel_stats": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.c_int]),
    "chai_cuda_buffer_alloc": (C.c_int, [P, C.c_uint64, C.c_size_t]),
    "chai_cuda_buffer_wrap": (C.c_int, [P, C.c_uint64, P, C.c_size_t]),
    "chai_cuda_buffer_info": (C.c_int, [P, C.c_uint64, C.POINTER(P), C.POINTER(C.c_size_t)]),
    "chai_cuda_upload": (C.c_int, [P, C.c_uint64, P, C.c_size_t]),
    "chai_cuda_readback": (C.c_int, [P, C.c_uint64, P, C.c_size_t]),
    "chai_cuda_release": (C.c_int, [P, C.c_uint64]),
    "chai_cuda_buffer_copy": (C.c_int, [P, C.c_uint64, C.c_uint64, C.c_size_t]),
    "chai_cuda_evaluate": (C.c_int, [P, C.POINTER(chai_trace_desc), C.POINTER(chai_buffer_binding), C.c_size_t]),
    "chai_cuda_trace_source": (C.c_int, [C.POINTER(chai_trace_desc), C.POINTER(chai_buffer_binding), C.c_size_t,
                                         C.c_char_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "chai_cuda_trace_shapes": (C.c_int, [C.POINTER(chai_trace_desc), C.POINTER(chai_buffer_binding), C.c_size_t,
                                         C.POINTER(chai_value_shape), C.c_size_t, C.POINTER(C.c_size_t)]),
    "chai_cuda_evaluate_many": (C.c_int, [P, C.POINTER(C.POINTER(chai_trace_desc)), C.c_size_t,
                                          C.POINTER(C.c_double)]),
    "chai_cuda_rng_fill": (C.c_int, [P, C.POINTER(chai_rng_desc), P]),
    "chai_cuda_gemm": (C.c_int, [P, C.POINTER(chai_gemm_desc)]),
    "chai_cuda_gemm_host": (C.c_int, [P, C.POINTER(chai_gemm_desc), C.c_int64]),
    "chai_cuda_gemv": (C.c_int, [P, C.c_uint32, C.c_int, C.c_int64, C.c_int64, C.c_double, P, C.c_int64, P,
                                 C.c_double, P]),
    "chai_cuda_gemm_grouped": (C.c_int, [P, C.c_int32, C.POINTER(chai_gemm_problem), C.c_int32]),
    "chai_cuda_reduce": (C.c_int, [P, C.c_uint32, C.c_uint32, P, P, C.c_uint64, C.c_uint32,
                                   C.POINTER(C.c_double)]),
    "chai_cuda_reduce_noalloc": (C.c_int, [C.c_uint32, C.c_uint32, P, P, C.c_uint64, C.c_uint32, P, P]),
    "chai_cuda_tune": (C.c_int, [P, C.POINTER(chai_gemm_key), C.c_int, C.POINTER(chai_gemm_cfg)]),
    "chai_cuda_tune_db_load": (C.c_int, [P, C.c_char_p]),
    "chai_cuda_tune_db_save": (C.c_int, [P, C.c_char_p]),
    "chai_cuda_tune_sweep": (C.c_int, [P, C.POINTER(chai_gemm_key), C.POINTER(chai_gemm_cfg), C.c_int,
                                       C.POINTER(C.c_int)]),
    "chai_cuda_tune_features": (C.c_int, [C.POINTER(chai_gemm_key), C.POINTER(chai_gemm_cfg),
                                          C.POINTER(C.c_float)]),
    "chai_cuda_mlp_train": (C.c_int, [P, C.POINTER(chai_gemm_key), C.POINTER(chai_gemm_cfg), C.c_size_t, C.c_int,
                                      C.c_double, C.c_uint64, C.POINTER(C.c_double)]),
    "chai_cuda_mlp_predict": (C.c_int, [P, C.POINTER(chai_gemm_key), C.POINTER(chai_gemm_cfg), C.c_size_t,
                                        C.POINTER(C.c_double)]),
    "chai_cuda_mlp_gradients": (C.c_int, [P, C.POINTER(chai_gemm_key), C.POINTER(chai_gemm_cfg), C.c_size_t,
                                          C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_double)]),
    "chai_cuda_mlp_weights": (C.c_int, [P, C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_size_t), C.c_int]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError("chai_b200: %s is missing -- run `python -m chai_b200.build` "
                               "(there is no CPU fallback)" % LIB_PATH)
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class ChaiError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        super().__init__("chai_b200 %s (%d): %s" % (ERR.get(status, "?"), status, detail))


def check(status: int, ctx=None) -> None:
    if status != CHAI_OK:
        detail = ""
        if ctx:
            d = lib().chai_cuda_last_error(ctx)
            detail = d.decode(errors="replace") if d else ""
        raise ChaiError(status, detail)
