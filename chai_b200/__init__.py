"""chai_b200: B200 (sm_100a) back end for chai traced array programs.

The product is the C-ABI shared library libchai_b200.so (include/chai_b200.h):
the trace translator, the fused trace kernel templates, GEMM/GEMV/reduction
kernels, the device memory manager and the GEMM tuner.  This package adds
  _lib   ctypes binding of every C-ABI entry point,
  api    a Python mirror of chai's array front end (api/chai.h) that records
         chai bytecode and evaluates traces through the C ABI,
  build  the in-tree build recipe (nvcc, -gencode arch=compute_100a,code=sm_100a).
"""
from . import _lib  # noqa: F401

__all__ = ["_lib", "api", "build"]
