"""The C-ABI library loads on a CPU-only machine, exports every entry point
include/chai_b200.h declares, and reports the absence of a GPU as a status
(no CPU fallback)."""
import ctypes as C
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "chai_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(chai_cuda_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "chai_cuda_evaluate" in names and "chai_cuda_init" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from chai_b200 import _lib
    lib = _lib.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(declared_functions()) <= set(_lib.SIGNATURES), "ctypes binding misses a declaration"


def test_nm_exports_match_header():
    so = ROOT / "chai_b200" / "libchai_b200.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (chai_cuda_\w+)", out))
    assert set(declared_functions()) <= exported


def test_error_strings():
    from chai_b200 import _lib
    lib = _lib.lib()
    assert lib.chai_cuda_error_string(0) == b"ok"
    assert b"device" in lib.chai_cuda_error_string(-7)


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU path")
def test_init_without_gpu_reports_no_device():
    from chai_b200 import _lib
    ctx = C.c_void_p()
    st = _lib.lib().chai_cuda_init(0, None, C.byref(ctx))
    assert st == -7 and not ctx.value


def test_fault_injection_on_init_is_host_side():
    """CHAI_FAULT_INJECT makes the named entry point fail before touching a GPU."""
    code = ("import ctypes as C, sys; sys.path.insert(0, %r); from chai_b200 import _lib; "
            "ctx = C.c_void_p(); print(_lib.lib().chai_cuda_init(0, None, C.byref(ctx)))" % str(ROOT))
    env = dict(os.environ, CHAI_FAULT_INJECT="init")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env).stdout.strip()
    assert out == "-9"


def test_null_arguments_are_invalid():
    from chai_b200 import _lib
    lib = _lib.lib()
    assert lib.chai_cuda_evaluate(None, None, None, 0) == -1
    assert lib.chai_cuda_shutdown(None) == -1
    assert lib.chai_cuda_readback(None, 1, None, 0) == -1


def test_c_consumer_struct_layout_matches_ctypes(tmp_path):
    """tests/abi_layout.c, compiled as C99 against include/chai_b200.h, prints
    every structure's size and field offsets; the ctypes binding must agree."""
    from chai_b200 import _lib
    exe = tmp_path / "abi_layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I" + str(ROOT / "include"),
                    str(ROOT / "tests" / "abi_layout.c"), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    checked = 0
    for ln in filter(None, lines):
        name, val = ln.split()
        if "." in name:
            struct, field = name.split(".")
            assert getattr(getattr(_lib, struct), field).offset == int(val), name
        else:
            assert C.sizeof(getattr(_lib, name)) == int(val), name
        checked += 1
    assert checked > 60


def test_trace_shapes_without_a_device():
    """chai_cuda_trace_shapes parses a trace and reports each assignment's
    value (needs no GPU): make2 of a 3 x 5 f32 box, then s = sum(A * A)."""
    from chai_b200 import _lib as L
    import chai_b200.api as ch
    cells_a = [ch._bc(L.BC_MEMORY, buffer=1), ch._sc(1), ch._sc(3), ch._sc(5), ch._op(66)]   # make2_f32
    cells_s = [ch._bc(L.BC_VARIABLE, 7, 0), ch._bc(L.BC_VARIABLE, 7, 0), ch._op(13), ch._op(132), ch._op(3)]   # sum(a * a) -> f32
    desc, keep = ch.build_desc([(7, 0, cells_a), (8, 0, cells_s)])
    out = (L.chai_value_shape * 4)()
    n = C.c_size_t(0)
    st = L.lib().chai_cuda_trace_shapes(C.byref(desc), None, 0, out, 4, C.byref(n))
    assert st == 0 and n.value == 2
    assert (out[0].variable, out[0].prec, out[0].width, out[0].height, out[0].slots) == (7, L.F32, 5, 3, 1)
    assert (out[1].variable, out[1].prec, out[1].width, out[1].height) == (8, L.F32, 1, 1)
