"""CPU oracle for chai's trace back end -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check in __graft_entry__.py and bench.py's CPU-baseline
leg may import this package.  It is the checker, never the thing measured or
shipped: the product (chai_b200) has no CPU path and fails loudly when its CUDA
library is missing.

Contents
  r123.c / r123.h   restatement of the reference JIT's Random123 generators and
                    chai's uniform / normal conversions (Random123/R123Philox.cpp,
                    Random123/R123Threefry.cpp, kernel/Function.cpp:388-503,
                    enqueue/EnqueueAST.cpp:496-545)
  ops.c             restatement of the interpreter's matmul / GEMV / reduction /
                    gather semantics (interp/InterpMatmulBase.hpp:25-61,
                    interp/InterpAccum.cpp:13-70, interp/InterpGather.hpp:19-44)
  build_ref.py      recipe compiling the reference's own interpreter and its
                    Random123 text from the reference sources into oracle/_ref/
  ref_driver.cpp    runs named traces through the reference interpreter
  ref.py            Python access to oracle/_ref (reference interpreter, pins)

Parity pins: the Random123 restatement is checked against the reference's
generated generator text and the vendored upstream Random123 text
(tests/test_oracle.py); the array-op restatement is checked against the reference
interpreter itself and against fixtures it produced (tests/golden/).
"""
from .cpu import *  # noqa: F401,F403
