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
  mlp.py            restatement of the tuner's cost model (features, MLP
                    forward / backward) for the GPU gradient check
  build_ref.py      recipe compiling the reference's own interpreter and its
                    Random123 text (bijections and chai's uniform / normal
                    wrappers) from the reference sources into oracle/_ref/
  ref_driver.cpp    runs named traces through the reference interpreter

Parity pins (tests/test_oracle.py): the Random123 restatement is checked
against the reference JIT's generated text -- bijections and every uniform /
normal wrapper -- and the vendored upstream Random123 text; the array-op
restatement against the reference interpreter itself (oracle/_ref, when built)
and against fixtures it produced (tests/golden/, made by
tests/golden/make_golden.py).
"""
from .cpu import *  # noqa: F401,F403
