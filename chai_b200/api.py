"""Host-side mirror of chai's array front end, driving the B200 back end.

This module records chai bytecode exactly as the reference front end does
(api/ArrayFP.cpp, api/ArrayFun.cpp, api/DuoFun.cpp, api/TriFun.cpp,
api/RngFun.cpp, api/IndexFun.cpp, api/MatmulFun.cpp push orders and opcode
numbers from bytecode/ByteCodes.hpp) and hands each trace to the CUDA back end
through the C ABI (chai_cuda_evaluate), the way the reference's scheduler hands
a VectorTrace to a DeviceBase.  Names follow api/chai.h: init/shutdown,
Arrayf32/Arrayf64/Arrayi32/Arrayu32, make1/make2, index_*, zeros_*/ones_*,
rng_uniform_make/rng_normal_make with RNGf32/RNGf64/RNGi32/RNGu32, matmul,
sum/mean/dot_product, cond, gather1_floor/gather2_floor, transpose, the math
functions, read_scalar/read1/read2.

A trace is scheduled at the first read-back, as in the reference
(api/ArrayFP.cpp:86-104).  Arrays that are still referenced from Python when a
trace runs stay resident in HBM (the reference's live variables); everything
else in the trace is fused into registers.

Python numbers follow C++ literal typing: a float is an f64 literal and an int
an i32 literal (DuoFun/TriFun overloads), so `0.2 * z` is computed in f64 and
rounded at the assignment, as the reference interpreter does.  Wrap a literal
in numpy.float32 to keep it f32.
"""
from __future__ import annotations

import builtins
import ctypes as C
import itertools
import weakref

import numpy as np

from . import _lib as L

# opcode numbers (bytecode/ByteCodes.hpp)
OPS1 = dict(acos=200, acosh=201, acospi=202, asin=203, asinh=204, asinpi=205, atan=206, atanh=208, atanpi=209,
            cbrt=211, ceil=212, cos=214, cosh=215, cospi=216, erfc=217, erf=218, exp=219, exp2=220, exp10=221,
            expm1=222, fabs=223, floor=225, ilogb=233, lgamma=235, log=237, log2=238, log10=239, log1p=240,
            logb=241, nan=246, rint=253, round=255, rsqrt=256, sin=257, sinh=259, sinpi=260, sqrt=261, tan=262,
            tanh=263, tanpi=264, tgamma=265, trunc=266, degrees=301, radians=305, sign=308, abs=400, clz=404,
            isfinite=507, isinf=508, isnan=509, isnormal=510, signbit=513)
OPS2 = dict(atan2=207, atan2pi=210, copysign=213, fdim=224, fmax=227, fmin=228, fmod=229, hypot=232, ldexp=234,
            maxmag=243, minmag=244, nextafter=247, pow=248, pown=249, powr=250, remainder=251, rootn=254,
            max=302, min=303, step=306, abs_diff=401, add_sat=402, hadd=405, mul24=411, mul_hi=412, rhadd=413,
            rotate=414, sub_sat=415, isequal=500, isnotequal=501, isgreater=502, isgreaterequal=503, isless=504,
            islessequal=505, islessgreater=506, isordered=511, isunordered=512)
OPS3 = dict(fma=226, mad=242, clamp=300, mix=304, smoothstep=307, mad24=406, mad_hi=407, mad_sat=408)

_max = builtins.max

_PREC_NAME = {L.U32: "u32", L.I32: "i32", L.F32: "f32", L.F64: "f64"}
_PREC_DTYPE = {L.U32: np.uint32, L.I32: np.int32, L.F32: np.float32, L.F64: np.float64}
_DTYPE_PREC = {np.dtype(np.uint32): L.U32, np.dtype(np.int32): L.I32, np.dtype(np.float32): L.F32,
               np.dtype(np.float64): L.F64}
_OFS = {L.U32: 0, L.I32: 1, L.F32: 2, L.F64: 3}


def _bc(kind, code=0, version=0, scalar=0.0, buffer=0):
    return (kind, code, version, scalar, buffer)


def _op(code):
    return _bc(L.BC_OPCODE, code)


def _sc(v):
    return _bc(L.BC_SCALAR, scalar=float(v))


# ------------------------------------------------------------------ device

class Device:
    """One back-end device: a chai_cuda_ctx (the CudaDevice plug-in instance)."""

    def __init__(self, device: int = 0, config: str | None = None):
        self.ctx = C.c_void_p()
        L.check(L.lib().chai_cuda_init(device, config.encode() if config else None, C.byref(self.ctx)))
        self._ids = itertools.count(1)
        self.kernel_launches = 0

    def close(self):
        if self.ctx:
            L.lib().chai_cuda_shutdown(self.ctx)
            self.ctx = C.c_void_p()

    def new_id(self) -> int:
        return next(self._ids)

    def upload(self, arr: np.ndarray) -> int:
        arr = np.ascontiguousarray(arr)
        bid = self.new_id()
        L.check(L.lib().chai_cuda_upload(self.ctx, bid, arr.ctypes.data_as(C.c_void_p), arr.nbytes), self.ctx)
        return bid

    def readback(self, bid: int, n: int, dtype) -> np.ndarray:
        out = np.empty(n, dtype=dtype)
        L.check(L.lib().chai_cuda_readback(self.ctx, bid, out.ctypes.data_as(C.c_void_p), out.nbytes), self.ctx)
        return out

    def release(self, bid: int):
        if self.ctx:
            L.lib().chai_cuda_release(self.ctx, bid)

    def evaluate(self, stmts, bindings, num_traces: int = 1, kernels=None):
        desc, keep = build_desc(stmts, num_traces, kernels)
        binds = (L.chai_buffer_binding * _max(1, len(bindings)))()
        for i, b in enumerate(bindings):
            binds[i] = L.chai_buffer_binding(*b)
        L.check(L.lib().chai_cuda_evaluate(self.ctx, C.byref(desc), binds, len(bindings)), self.ctx)


def build_desc(stmts, num_traces=1, kernels=None):
    """chai_trace_desc from [(lhs_var, lhs_ver, [cells...]), ...] and the
    trace's inline kernels [(source, name, [(kind, prec, var, ver, value)],
    (g0, g1), (l0, l1)), ...]."""
    arr = (L.chai_stmt * _max(1, len(stmts)))()
    keep = [arr]
    for i, (var, ver, cells) in enumerate(stmts):
        ca = (L.chai_bc * len(cells))()
        for j, (kind, code, version, scalar, buffer) in enumerate(cells):
            ca[j] = L.chai_bc(kind, code, version, 0, scalar, buffer)
        keep.append(ca)
        arr[i] = L.chai_stmt(var, ver, len(cells), 0, ca)
    desc = L.chai_trace_desc(num_traces, len(stmts), arr, 0)
    if kernels:
        ka = (L.chai_inline_kernel * len(kernels))()
        for i, (src, name, args, gsize, lsize) in enumerate(kernels):
            aa = (L.chai_kernel_arg * _max(1, len(args)))()
            for j, (kind, prec, var, ver, value) in enumerate(args):
                aa[j] = L.chai_kernel_arg(kind, prec, var, ver, float(value))
            sb, nb = src.encode(), name.encode()
            keep += [aa, sb, nb]
            ka[i] = L.chai_inline_kernel(sb, nb, len(args), 0, aa, (C.c_uint64 * 2)(*gsize),
                                         (C.c_uint64 * 2)(*lsize))
        keep.append(ka)
        desc.kernels = ka
        desc.n_kernels = len(kernels)
    keep.append(desc)
    return desc, keep


_vm: Device | None = None


def init(config: str | None = None, device: int = 0) -> Device:
    """chai::init (api/ManageVM.cpp:16-25)."""
    global _vm
    if _vm is None:
        _vm = Device(device, config)
    return _vm


def shutdown():
    """chai::shutdown: evaluate nothing further, free every device buffer."""
    global _vm
    if _vm is not None:
        _Client.pending.clear()
        _Client.keep = []
        _vm.close()
        _vm = None


def vm() -> Device:
    if _vm is None:
        raise RuntimeError("chai_b200: call init() first")
    return _vm


# ------------------------------------------------------------------ trace client

class _Client:
    """The per-thread trace (common/ClientTrace.hpp): statements since the last
    read-back, and the arrays that own device buffers."""
    pending: list = []            # (lhs_var, lhs_ver, cells, owner array or None)
    keep: list = []               # make1/make2 arrays whose host data the trace reads
    kernels: list = []            # inline OpenCL kernels of the pending trace
    vars = itertools.count(1)


def _schedule():
    """Evaluate the pending trace (Scheduler::wait -> DeviceBase::evaluate)."""
    dev = vm()
    stmts = _Client.pending
    kernels = _Client.kernels
    _Client.pending = []
    _Client.kernels = []
    if not stmts:
        return
    assigned = {}
    referenced = set()
    for var, ver, cells, owner in stmts:
        for c in cells:
            if c[0] == L.BC_VARIABLE:
                referenced.add(c[1])
        if owner is not None:
            assigned[var] = owner
    for _, _, args, _, _ in kernels:
        for kind, _, var, _, _ in args:
            if kind == L.KARG_ARRAY:
                referenced.add(var)
    bindings = []
    # inputs: arrays from earlier traces referenced here
    for var in referenced:
        if var in assigned:
            continue
        a = Array._registry.get(var)
        a = a() if a is not None else None
        if a is None or a._buffer is None:
            raise RuntimeError("chai_b200: variable %d has no value" % var)
        bindings.append((var, a.prec, a.W, a.H, a.slots, 0, a._buffer))
    # outputs: arrays assigned here that are still alive
    for var, owner in assigned.items():
        a = owner()
        if a is None:
            continue
        if a._buffer is None:
            a._buffer = dev.new_id()
            weakref.finalize(a, _release, a._buffer)
        bindings.append((var, a.prec, a.W, a.H, a.slots, 0, a._buffer))
    try:
        dev.evaluate([(v, ver, cells) for v, ver, cells, _ in stmts], bindings, kernels=kernels)
    finally:
        _Client.keep = []


def _release(bid):
    if _vm is not None:
        _vm.release(bid)


# ------------------------------------------------------------------ expressions

def _lit(v) -> "ArrayExp":
    if isinstance(v, ArrayExp):
        return v
    if isinstance(v, (np.floating,)) and np.dtype(type(v)) == np.float32:
        return _Scalar(float(v), L.F32)
    if isinstance(v, (float, np.floating)):
        return _Scalar(float(v), L.F64)
    if isinstance(v, (np.unsignedinteger,)):
        return _Scalar(int(v), L.U32)
    if isinstance(v, (int, np.integer, bool)):
        return _Scalar(int(v), L.I32)
    raise TypeError("unsupported literal %r" % (v,))


class ArrayExp:
    """An array expression (api/chai.h ArrayExp): pushes its bytecode."""
    __array_ufunc__ = None     # numpy scalars defer to our reflected operators
    prec = L.F32
    W = H = slots = 1

    def cells(self, out: list):
        raise NotImplementedError

    # arithmetic (DuoFun with operator codes, api/OpsDuoFun.cpp)
    def __add__(self, o): return _Fun(11, self, o)
    def __radd__(self, o): return _Fun(11, o, self)
    def __sub__(self, o): return _Fun(14, self, o)
    def __rsub__(self, o): return _Fun(14, o, self)
    def __mul__(self, o): return _Fun(13, self, o)
    def __rmul__(self, o): return _Fun(13, o, self)
    def __truediv__(self, o): return _Fun(12, self, o)
    def __rtruediv__(self, o): return _Fun(12, o, self)
    def __mod__(self, o): return _Fun(17, self, o)
    def __lshift__(self, o): return _Fun(18, self, o)
    def __rshift__(self, o): return _Fun(19, self, o)
    def __and__(self, o): return _Fun(20, self, o)
    def __or__(self, o): return _Fun(21, self, o)
    def __xor__(self, o): return _Fun(22, self, o)
    def __eq__(self, o): return _Fun(32, self, o)
    def __ne__(self, o): return _Fun(33, self, o)
    def __ge__(self, o): return _Fun(34, self, o)
    def __gt__(self, o): return _Fun(35, self, o)
    def __le__(self, o): return _Fun(36, self, o)
    def __lt__(self, o): return _Fun(37, self, o)
    def __neg__(self): return _Fun(10, self)
    def __invert__(self): return _Fun(15, self)
    __hash__ = object.__hash__


class _Scalar(ArrayExp):
    def __init__(self, v, prec):
        self.v, self.prec = v, prec

    def cells(self, out):
        out.append(_sc(self.v))
        out.append(_op(5 + _OFS[self.prec]))


class _Fun(ArrayExp):
    """ArrayFun / DuoFun / TriFun: arguments pushed last-first, then the code."""

    def __init__(self, code, *args, dims="max"):
        self.code = code
        self.args = [_lit(a) for a in args]
        ps = [a.prec for a in (self.args[1:] if code == 23 else self.args)]
        self.prec = _max(ps) if ps else L.F32
        if 200 <= code <= 299 or code in (301, 304, 305, 306, 307, 308) or 506 <= code <= 513:
            self.prec = _max(self.prec, L.F32)
        if dims == "first":
            a = self.args[0]
            self.W, self.H = a.W, a.H
            self.slots = _max(x.slots for x in self.args)
        elif dims == "reduced":
            self.W = self.H = 1
            self.slots = self.args[0].slots
        else:
            self.W = _max(a.W for a in self.args)
            self.H = _max(a.H for a in self.args)
            self.slots = _max(a.slots for a in self.args)

    def cells(self, out):
        for a in reversed(self.args):
            a.cells(out)
        out.append(_op(self.code))


class _Raw(ArrayExp):
    """A leaf with a fixed bytecode list (index, rng, make, zeros)."""

    def __init__(self, cells, prec, W, H, slots=1):
        self._cells, self.prec, self.W, self.H, self.slots = cells, prec, W, H, slots

    def cells(self, out):
        out.extend(self._cells)


class _Matmul(ArrayExp):
    def __init__(self, a, b, c=None, alpha=1.0, beta=1.0):
        self.a, self.b, self.c = _lit(a), _lit(b), (None if c is None else _lit(c))
        self.alpha, self.beta = alpha, beta
        self.prec = _max(self.a.prec, self.b.prec)
        self.slots = _max(self.a.slots, self.b.slots)
        l, r = self.a, self.b
        if self.c is not None:
            self.W, self.H = self.c.W, self.c.H
        elif l.H == 1 and r.H == 1:
            self.W, self.H = r.W, l.W
        elif l.H == 1:
            self.W, self.H = r.W, 1
        elif r.H == 1:
            self.W, self.H = l.H, 1
        else:
            self.W, self.H = r.W, l.H

    def cells(self, out):
        if self.c is None:                      # ArrayFun(matmul, A, B)
            self.b.cells(out)
            self.a.cells(out)
            out.append(_op(120))
        else:                                   # MatmulFun (api/MatmulFun.cpp:26-35)
            out.append(_sc(self.beta))
            out.append(_sc(self.alpha))
            self.c.cells(out)
            self.b.cells(out)
            self.a.cells(out)
            out.append(_op(121))


class Array(ArrayExp):
    """Arrayu32 / Arrayi32 / Arrayf32 / Arrayf64 (api/ArrayFP.cpp)."""
    _registry: dict = {}
    PREC = L.F32

    def __init__(self, rhs=None, *, _raw=None):
        self.prec = self.PREC
        self.var = next(_Client.vars)
        self.version = 1
        self._buffer = None
        Array._registry[self.var] = weakref.ref(self)
        if _raw is not None:
            cells, W, H, slots = _raw
            self.W, self.H, self.slots = W, H, slots
            self._assign(list(cells), convert=False)
        elif rhs is not None:
            rhs = _lit(rhs)
            self.W, self.H, self.slots = rhs.W, rhs.H, rhs.slots
            out = []
            rhs.cells(out)
            self._assign(out, convert=True)

    def _assign(self, cells, convert):
        if convert:
            cells.append(_op(1 + _OFS[self.prec]))
        _Client.pending.append((self.var, self.version, cells, weakref.ref(self)))
        self.version += 1

    def assign(self, rhs):
        """operator= (api/ArrayFP.cpp:46-53)."""
        rhs = _lit(rhs)
        out = []
        rhs.cells(out)
        self.W, self.H, self.slots = rhs.W, rhs.H, rhs.slots
        self._assign(out, convert=True)
        return self

    def cells(self, out):
        # a value from an earlier trace stays alive (with its device buffer)
        # until the pending trace that reads it has run, as the reference's
        # client trace holds its operands (common/ClientTrace.cpp RefSet)
        if self._buffer is not None:
            _Client.keep.append(self)
        out.append(_bc(L.BC_VARIABLE, self.var, self.version - 1))

    # read-backs (api/ArrayFP.cpp:86-228)
    def _read(self, code_base, n):
        dev = vm()
        bid = dev.new_id()
        cells = [_bc(L.BC_MEMORY, buffer=bid), _bc(L.BC_VARIABLE, self.var, self.version - 1),
                 _op(code_base + _OFS[self.prec])]
        _Client.pending.append((self.var, self.version, cells, None))
        _schedule()
        out = dev.readback(bid, n, _PREC_DTYPE[self.prec])
        dev.release(bid)
        return out

    def read_scalar(self):
        """Host sum of the vector partials, as the reference client does."""
        vl = 2 if self.prec == L.F64 else 4
        parts = self._read(90, vl * self.slots).reshape(self.slots, vl)
        s = parts[:, 0].copy()
        for j in range(1, vl):
            s = s + parts[:, j]
        return s[0] if self.slots == 1 else s

    def read1(self):
        return self._read(94, self.W * self.H * self.slots)

    def read2(self):
        a = self._read(98, self.W * self.H * self.slots)
        return a.reshape(self.slots, self.H, self.W) if self.slots > 1 else a.reshape(self.H, self.W)


class Arrayu32(Array):
    PREC = L.U32


class Arrayi32(Array):
    PREC = L.I32


class Arrayf32(Array):
    PREC = L.F32


class Arrayf64(Array):
    PREC = L.F64


_ARR = {L.U32: Arrayu32, L.I32: Arrayi32, L.F32: Arrayf32, L.F64: Arrayf64}


# ------------------------------------------------------------------ creation

def make1(data, W=None):
    data = np.ascontiguousarray(data)
    prec = _DTYPE_PREC[data.dtype]
    slots = 1 if data.ndim == 1 else data.shape[0]
    W = W or data.shape[-1]
    bid = vm().upload(data)
    cells = [_bc(L.BC_MEMORY, buffer=bid), _sc(slots), _sc(1), _sc(W), _op(60 + _OFS[prec])]
    a = _ARR[prec](_raw=(cells, W, 1, slots))
    a._buffer = bid
    weakref.finalize(a, _release, bid)
    _Client.keep.append(a)
    return a


def make2(data):
    """make2(W, H, cpu) from an (H, W) or (slots, H, W) array."""
    data = np.ascontiguousarray(data)
    prec = _DTYPE_PREC[data.dtype]
    slots = 1 if data.ndim == 2 else data.shape[0]
    H, W = data.shape[-2], data.shape[-1]
    bid = vm().upload(data)
    cells = [_bc(L.BC_MEMORY, buffer=bid), _sc(slots), _sc(H), _sc(W), _op(64 + _OFS[prec])]
    a = _ARR[prec](_raw=(cells, W, H, slots))
    a._buffer = bid
    weakref.finalize(a, _release, bid)
    _Client.keep.append(a)
    return a


def _index(prec, dim, W, H=None):
    if H is None:
        return _Raw([_sc(W), _sc(dim), _op(42 + _OFS[prec])], prec, W, 1)
    return _Raw([_sc(H), _sc(W), _sc(dim), _op(46 + _OFS[prec])], prec, W, H)


def index_u32(dim, W, H=None): return _index(L.U32, dim, W, H)
def index_i32(dim, W, H=None): return _index(L.I32, dim, W, H)
def index_f32(dim, W, H=None): return _index(L.F32, dim, W, H)
def index_f64(dim, W, H=None): return _index(L.F64, dim, W, H)


def _fill(prec, one, W, H=None):
    if H is None:
        code = (68 if one else 76) + _OFS[prec]
        return _Raw([_sc(W), _op(code)], prec, W, 1)
    code = (72 if one else 80) + _OFS[prec]
    if prec == L.F64 and not one:
        code = 73     # zeros2_f64 (bytecode/ByteCodes.hpp:105)
    return _Raw([_sc(H), _sc(W), _op(code)], prec, W, H)


def zeros_f32(W, H=None): return _fill(L.F32, False, W, H)
def zeros_f64(W, H=None): return _fill(L.F64, False, W, H)
def ones_f32(W, H=None): return _fill(L.F32, True, W, H)
def ones_f64(W, H=None): return _fill(L.F64, True, W, H)
def zeros_i32(W, H=None): return _fill(L.I32, False, W, H)
def zeros_u32(W, H=None): return _fill(L.U32, False, W, H)
def ones_u32(W, H=None): return _fill(L.U32, True, W, H)


# ------------------------------------------------------------------ RNG

RNG_PHILOX, RNG_THREEFRY = L.PHILOX, L.THREEFRY
RNG_DEFAULT = RNG_PHILOX          # api/chai.h:416


class _RNG:
    """RNGBase32 / RNGBase64 (api/RNGBase.cpp): variant and running seed."""
    PREC = L.F32
    BITS = 32

    def __init__(self, variant=RNG_PHILOX, seed=0):
        self.variant = variant
        self.seed = int(seed)

    def _inc(self, n):
        self.seed = (self.seed + n) & ((1 << self.BITS) - 1)


class RNGf32(_RNG):
    PREC = L.F32


class RNGi32(_RNG):
    PREC = L.I32


class RNGu32(_RNG):
    PREC = L.U32


class RNGf64(_RNG):
    PREC = L.F64
    BITS = 64


def rng_uniform_make(g: _RNG, W, H=1, slots=1, min_limit=None, max_limit=None):
    """api/RngFun.cpp:15-90; f32/f64 take limits (u * (max-min) + min)."""
    cells = []
    if g.PREC in (L.F32, L.F64):
        if min_limit is None:
            min_limit, max_limit = 0.0, 1.0
        cells += [_sc(max_limit), _sc(min_limit)]
        code = 114 if g.PREC == L.F32 else 115
    else:
        code = 112 if g.PREC == L.U32 else 113
    cells += [_sc(slots), _sc(H), _sc(W), _sc(g.seed), _sc(g.variant), _op(code)]
    g._inc(W * H * slots)
    return _Raw(cells, g.PREC, W, H, slots)


def rng_normal_make(g: _RNG, W, H=1, slots=1):
    code = 110 if g.PREC == L.F32 else 111
    cells = [_sc(slots), _sc(H), _sc(W), _sc(g.seed), _sc(g.variant), _op(code)]
    g._inc(W * H * slots)
    return _Raw(cells, g.PREC, W, H, slots)


# ------------------------------------------------------------------ functions

def _mk1(code):
    return lambda a: _Fun(code, a)


def _mk2(code):
    return lambda a, b: _Fun(code, a, b)


def _mk3(code):
    return lambda a, b, c: _Fun(code, a, b, c)


for _n, _c in OPS1.items():
    globals()[_n] = _mk1(_c)
for _n, _c in OPS2.items():
    globals()[_n] = _mk2(_c)
for _n, _c in OPS3.items():
    globals()[_n] = _mk3(_c)


def cond(pred, a, b):
    """TriFun(operatorCONDEXPR, pred, a, b) (api/OpsCond.cpp)."""
    return _Fun(23, pred, a, b)


def logical_and(a, b): return _Fun(30, a, b)
def logical_or(a, b): return _Fun(31, a, b)
def logical_not(a): return _Fun(16, a)


def convert_f32(a): return _Fun(3, a)
def convert_f64(a): return _Fun(4, a)
def convert_i32(a): return _Fun(2, a)
def convert_u32(a): return _Fun(1, a)


def sum(a): return _Fun(132, a, dims="reduced")             # noqa: A001
def mean(a): return _Fun(131, a, dims="reduced")
def dot_product(a, b): return _Fun(130, a, b, dims="reduced")
def gather1_floor(a, x): return _Fun(40, a, x, dims="first")
def gather2_floor(a, x, y): return _Fun(41, a, x, y, dims="first")


def transpose(a):
    f = _Fun(122, a)
    f.W, f.H = _lit(a).H, _lit(a).W
    return f


def matmul(a, b, c=None, alpha=1.0, beta=1.0):
    return _Matmul(a, b, c, alpha, beta)


# ------------------------------------------------------------------ inline OpenCL

_CL_SCALARS = {"unsigned": L.U32, "uint": L.U32, "int": L.I32, "float": L.F32, "double": L.F64}
_CL_BYTES = {"char": 1, "uchar": 1, "short": 2, "ushort": 2, "int": 4, "uint": 4, "long": 8, "ulong": 8,
             "float": 4, "double": 8}


def _cl_vector_bytes(tok):
    """Bytes of one element of an OpenCL vector type name (a 3-vector is
    stored as a 4-vector), or 0 when `tok` names no vector type."""
    import re
    m = re.fullmatch(r"(char|uchar|short|ushort|int|uint|long|ulong|float|double)(2|3|4|8|16)", tok)
    if not m:
        return 0
    n = int(m.group(2))
    return _CL_BYTES[m.group(1)] * (4 if n == 3 else n)


def _cl_kernel_heads(text):
    """(name, parameter text) of every `__kernel void NAME(...)`; attributes
    between `__kernel` and `void` are skipped, as api/ProgramCL.cpp:156-177
    skips every token up to `void`."""
    import re
    out = []
    for m in re.finditer(r"\b(?:__kernel|kernel)\b", text):
        i = m.end()
        while True:
            while i < len(text) and text[i].isspace():
                i += 1
            if not text.startswith("__attribute__", i):
                break
            j = text.find("(", i)
            if j < 0:
                return out
            depth = 0
            for k in range(j, len(text)):
                depth += {"(": 1, ")": -1}.get(text[k], 0)
                if depth == 0:
                    break
            i = k + 1
        h = re.match(r"void\s+(\w+)\s*\(([^)]*)\)", text[i:])
        if h:
            out.append((h.group(1), h.group(2)))
    return out


def _cl_vector_params(text):
    """Per kernel, for each parameter: the element bytes of a vector-typed
    parameter (0 for the others)."""
    return {name: [_max([_cl_vector_bytes(t) for t in p.replace("*", " ").split()] or [0])
                   for p in params.split(",") if p.split()]
            for name, params in _cl_kernel_heads(text)}


def _cl_signatures(text):
    """Argument kinds and precisions of every `__kernel void NAME(...)` in the
    program text, as api/ProgramCL.cpp:45-176 reads them: __global / global /
    image2d_t parameters are arrays, __local / local ones local memory, the
    rest scalars; the precision is the parameter's uint / unsigned / int /
    float / double keyword."""
    sigs = {}
    for name, params in _cl_kernel_heads(text):
        args = []
        for p in params.split(","):
            toks = p.replace("*", " ").split()
            if not toks:
                continue
            if any(t in ("__global", "global", "image2d_t") for t in toks):
                kind = L.KARG_ARRAY
            elif any(t in ("__local", "local") for t in toks):
                kind = L.KARG_LOCAL
            else:
                kind = L.KARG_SCALAR
            prec = next((_CL_SCALARS[t] for t in toks if t in _CL_SCALARS), -1)
            args.append((kind, prec))
        sigs[name] = args
    return sigs


class ProgramCL:
    """Inline OpenCL kernels (api/chai.h ProgramCL).  The C++ form
    `(prog, "name", A, 1.5f)(N, 1)` is written `prog("name", A, f32(1.5))(N, 1)`:
    array arguments are updated in place, and later statements see the new
    values; the kernel runs in statement order within the trace."""

    def __init__(self, text):
        self.text = text if isinstance(text, str) else "\n".join(text)
        self._sigs = _cl_signatures(self.text)
        self._vbytes = _cl_vector_params(self.text)

    def __call__(self, name, *args):
        if name not in self._sigs:
            raise ValueError("ProgramCL: no __kernel named %r" % name)
        return _KernelCall(self, name, args)


class _KernelCall:
    def __init__(self, prog, name, args):
        self.prog, self.name, self.args = prog, name, args

    def __call__(self, *ws):
        """(global0, local0) or (global0, global1, local0, local1)."""
        if len(ws) == 2:
            gsize, lsize = (ws[0], 0), (ws[1], 0)
        elif len(ws) == 4:
            gsize, lsize = (ws[0], ws[1]), (ws[2], ws[3])
        else:
            raise TypeError("work space: (global0, local0) or (global0, global1, local0, local1)")
        sig = self.prog._sigs[self.name]
        if len(sig) != len(self.args):
            raise TypeError("ProgramCL: %s takes %d arguments" % (self.name, len(sig)))
        args = []
        vbytes = self.prog._vbytes.get(self.name, [0] * len(sig))
        for (kind, prec), vb, a in zip(sig, vbytes, self.args):
            if kind == L.KARG_ARRAY:
                if not isinstance(a, Array):
                    raise TypeError("ProgramCL: array arguments must be array variables")
                args.append((kind, a.prec, a.var, a.version - 1, 0.0))
                _Client.keep.append(a)
            elif vb and kind != L.KARG_LOCAL:
                raise TypeError("ProgramCL: %s: vector-typed scalar arguments are not supported" % self.name)
            else:
                args.append((kind, prec if prec >= 0 else L.F32, 0, 0, float(a)))
        idx = len(_Client.kernels)
        _Client.kernels.append((self.prog.text, self.name, args, gsize, lsize))
        var = next(_Client.vars)
        _Client.pending.append((var, 1, [_bc(L.BC_KERNEL, buffer=idx), _op(50)], None))


# ------------------------------------------------------------------ many traces

def record(build):
    """Record the statements `build()` creates without evaluating them; returns
    (statements, value of build()).  The statements form one trace."""
    saved = _Client.pending
    _Client.pending = []
    try:
        out = build()
        stmts = [(v, ver, cells) for v, ver, cells, _ in _Client.pending]
    finally:
        _Client.pending = saved
    return stmts, out


def evaluate_many(traces):
    """Evaluate many recorded traces that share one program (same bytecode
    up to scalar values: shapes, seeds, literals) and end in a reduction; one
    result per trace (chai_cuda_evaluate_many)."""
    dev = vm()
    keep = []
    ptrs = (C.POINTER(L.chai_trace_desc) * len(traces))()
    for i, stmts in enumerate(traces):
        desc, k = build_desc(stmts)
        keep.append((desc, k))
        ptrs[i] = C.pointer(desc)
    res = (C.c_double * len(traces))()
    L.check(L.lib().chai_cuda_evaluate_many(dev.ctx, ptrs, len(traces), res), dev.ctx)
    return np.frombuffer(res, dtype=np.float64).copy()
