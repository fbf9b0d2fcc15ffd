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
