"""Trace translator on the CPU: bytecode recorded by the front-end mirror is
planned, emitted as CUDA C and compiled with NVRTC for sm_100a
(chai_cuda_trace_source needs no device).  Checks fusion decisions and the
shape / precision rules."""
import ctypes as C

import numpy as np
import pytest

import chai_b200.api as ch
from chai_b200 import _lib as L

f32 = np.float32


def record(build):
    """Run `build()` against a fresh pending trace; return its statements."""
    ch._Client.pending = []
    keep = build()
    stmts = [(v, ver, cells) for v, ver, cells, _ in ch._Client.pending]
    ch._Client.pending = []
    return stmts, keep


def source(stmts, binds=(), config=None):
    desc, keep = ch.build_desc(stmts)
    b = (L.chai_buffer_binding * max(1, len(binds)))()
    for i, x in enumerate(binds):
        b[i] = L.chai_buffer_binding(*x)
    buf = C.create_string_buffer(1 << 21)
    need = C.c_size_t()
    st = L.lib().chai_cuda_trace_source(C.byref(desc), b, len(binds), config.encode() if config else None, buf,
                                        len(buf), C.byref(need))
    return st, buf.value.decode()


def read_stmt(arr, bid=99):
    return (arr.var, arr.version, [ch._bc(L.BC_MEMORY, buffer=bid), ch._bc(L.BC_VARIABLE, arr.var, arr.version - 1),
                                   ch._op(90 + ch._OFS[arr.prec])])


def test_monte_carlo_is_one_fused_kernel():
    def build():
        g = ch.RNGf32(ch.RNG_PHILOX, 42)
        return ch.Arrayf32(ch.mean(ch.max(f32(100) * ch.exp(f32(0.03) + f32(0.2) * ch.rng_normal_make(g, 8192, 16384))
                                          - f32(100), f32(0))))
    stmts, p = record(build)
    st, src = source(stmts + [read_stmt(p)])
    assert st == 0, src
    assert src.count("__global__") == 1          # RNG, exp, max and mean fused; result is the reduction
    assert "raw32<1230, 0>" in src and "box_muller_f32" in src and "block_sum" in src
    assert "double" not in src.split("for (long long c")[1].split("red[0] +=")[0].replace("(double)", "")


def test_reduce_accum_f32_option():
    """ReduceAccum=f32: per-thread partial sums of f32 reductions in f32, the
    block tree and the combine in FP64; the default accumulates in FP64."""
    def build():
        a = ch.index_f32(0, 64, 4)
        return ch.Arrayf32(ch.sum(a) + ch.dot_product(a, a))
    stmts, p = record(build)
    st, src = source(stmts + [read_stmt(p)])
    assert st == 0 and "redf" not in src and "red[0] += (double)v" in src
    st, src = source(stmts + [read_stmt(p)], config="ReduceAccum=f32")
    assert st == 0 and "redf[0] += v" in src and "red[1] = (double)redf[1];" in src


def test_double_literal_promotes_to_f64():
    def build():
        return ch.Arrayf32(0.2 * ch.index_f32(0, 64, 4) + 1.0)
    stmts, a = record(build)
    st, src = source(stmts, [(a.var, 4, 64, 4, 1, 0, 5)])
    assert st == 0, src
    assert "f2<13, double>" in src and "(float)v" in src


def test_kirsch_trace_is_one_kernel_with_gathers():
    from tests.test_gpu_trace import kirsch_expr

    def build():
        A = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(64), ch._sc(64), ch._op(66)], 64, 64, 1))
        return A, ch.Arrayf32(kirsch_expr(ch, A, 64, 64))
    stmts, (A, K) = record(build)
    st, src = source(stmts, [(K.var, 4, 64, 64, 1, 0, 8)])
    assert st == 0, src
    # every gather is a constant-offset stencil: one 2-D tiled kernel, the
    # source tile staged in shared memory by TMA (wrapped loads at borders)
    assert src.count("__global__") == 1 and src.count("gather_index") == 0
    assert "tma_load_3d(tile0" in src
    # the 8 gathers read 3 row windows (row offsets -1, 0, +1), each one
    # 16-byte shared load plus two edge elements
    assert src.count("const float* rowp = tile0") == 3 and src.count("chai_k::lds_vec(rowp") == 3
    # the max tree of 8 * s_k - 3 * total runs as 8 * max(s_k) - 3 * total
    # when 3 * total is finite (the plain tree otherwise, and with FuseMaxAffine=0)
    assert src.count("isinf(") == 1 and src.count("f2<13, float>") == 10   # 3 * total, fast, 8 slow
    st0, src0 = source(stmts, [(K.var, 4, 64, 64, 1, 0, 8)], "FuseMaxAffine=0")
    assert st0 == 0 and "isinf(" not in src0
    # a 64 x 64 image is smaller than one staged tile: its border tiles are
    # wrapped loads only
    assert "if (!interior && tile_ok)" not in src
    # two rows x 4 columns per thread: 4 row windows (offsets -1 .. +2) serve both rows
    st2, src2 = source(stmts, [(K.var, 4, 64, 64, 1, 0, 8)], "StencilRowsPerThread=2")
    assert st2 == 0 and src2.count("const float* rowp = tile0") == 4 and src2.count("chai_k::lds_vec(rowp") == 4
    assert "[8];" in src2 and " < H) chai_k::st4p(o" in src2 and "st4p" not in src
    # the index arithmetic under the stencil gathers is not emitted; f32 ops
    # stay scalar in stencil kernels
    body = src.split("chai_group")[1]
    assert "% 64)" not in body and "f2x4" not in body


def test_stencil_tile_height_follows_shared_memory_and_grid():
    """Stencil tiles are 64 rows tall when the staged tiles fit the 46 KiB of
    static shared memory and the image gives every SM four tiles; 32 rows
    otherwise (f64 sources, small images); StencilRows overrides."""
    from tests.test_gpu_trace import kirsch_expr

    def src_for(W, H, prec, cfg=None):
        def build():
            A = ch._ARR[prec](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(W), ch._sc(H),
                                     ch._op(66 if prec == L.F32 else 67)], W, H, 1))
            arr = ch.Arrayf32 if prec == L.F32 else ch.Arrayf64
            return A, arr(kirsch_expr(ch, A, W, H))
        stmts, (A, K) = record(build)
        st, src = source(stmts, [(K.var, prec, W, H, 1, 0, 8)], cfg)
        assert st == 0, src
        return src
    assert "blockIdx.y * 64" in src_for(8192, 8192, L.F32)
    assert "blockIdx.y * 32" in src_for(8192, 8192, L.F64)        # (64 + 2) x 136 x 8 B > 46 KiB
    assert "blockIdx.y * 32" in src_for(256, 256, L.F32)          # 2 x 4 tiles of 64 rows < 4 per SM
    assert "blockIdx.y * 16" in src_for(8192, 8192, L.F32, "StencilRows=16")


def test_flat_kernel_packs_f32_add_sub():
    """Element-wise kernels issue f32 add / sub as f32x2 pairs of neighbouring
    elements (registers of one 16-byte load); PackF32=0 keeps them scalar."""
    def build():
        a = ch.index_f32(0, 64, 4)
        return ch.Arrayf32((a + f32(1)) * f32(3) - a)
    stmts, a = record(build)
    st, src = source(stmts, [(a.var, 4, 64, 4, 1, 0, 5)])
    assert st == 0 and "f2x4<11>" in src and "f2x4<14>" in src and "f2x4<13>" not in src
    st0, src0 = source(stmts, [(a.var, 4, 64, 4, 1, 0, 5)], "PackF32=0")
    assert st0 == 0 and "f2x4" not in src0.split("chai_group")[1]


def test_data_dependent_gather_stays_generic():
    def build():
        A = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(64), ch._sc(64), ch._op(66)], 64, 64, 1))
        X = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=9), ch._sc(1), ch._sc(64), ch._sc(64), ch._op(66)], 64, 64, 1))
        return A, X, ch.Arrayf32(ch.gather2_floor(A, X, ch.index_f32(1, 64, 64)))
    stmts, (A, X, G) = record(build)
    st, src = source(stmts, [(G.var, 4, 64, 64, 1, 0, 8)])
    assert st == 0, src
    assert src.count("gather_index") == 2 and "tma_load_3d(" not in src.split("chai_group")[1]


def test_gather_of_value_computed_in_trace_splits_kernels():
    def build():
        a = ch.Arrayf32(ch.index_f32(0, 32, 32) * f32(2))
        return a, ch.Arrayf32(ch.gather2_floor(a, ch.index_f32(0, 32, 32) + f32(1), ch.index_f32(1, 32, 32)))
    stmts, (a, b) = record(build)
    st, src = source(stmts, [(b.var, 4, 32, 32, 1, 0, 9)])
    assert st == 0, src
    assert src.count("__global__") == 2


@pytest.mark.parametrize("prec", [0, 1, 4, 8])
def test_all_element_ops_compile(prec):
    """Every opcode family of the fused kernel compiles for every precision it
    accepts (int-only ops on u32/i32, fp-only ops on f32/f64)."""
    dt = {0: np.uint32, 1: np.int32, 4: np.float32, 8: np.float64}[prec]
    lit = dt(3)

    def build():
        x = ch._ARR[prec](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(8), ch._sc(16),
                                 ch._op(64 + ch._OFS[prec])], 16, 8, 1))
        outs = [x]
        if prec in (4, 8):
            for name in ch.OPS1:
                if name in ("clz", "abs"):
                    continue
                outs.append(ch._ARR[prec](getattr(ch, name)(x)))
            for name in ("atan2", "atan2pi", "copysign", "fdim", "fmax", "fmin", "fmod", "hypot", "maxmag", "minmag",
                         "nextafter", "pow", "pown", "powr", "remainder", "rootn", "max", "min", "step", "isequal",
                         "islessgreater", "isordered", "isunordered"):
                outs.append(ch._ARR[prec](getattr(ch, name)(x, lit)))
            for name in ("fma", "mad", "clamp", "mix", "smoothstep"):
                outs.append(ch._ARR[prec](getattr(ch, name)(x, lit, x)))
        else:
            for op in (x + lit, x - lit, x * lit, x / lit, x % lit, x << lit, x >> lit, x & lit, x | lit, x ^ lit,
                       ~x, -x, ch.abs(x), ch.clz(x), ch.abs_diff(x, lit), ch.add_sat(x, lit), ch.hadd(x, lit),
                       ch.mul24(x, lit), ch.mul_hi(x, lit), ch.rhadd(x, lit), ch.rotate(x, lit), ch.sub_sat(x, lit),
                       ch.mad24(x, lit, x), ch.mad_hi(x, lit, x), ch.mad_sat(x, lit, x), ch.max(x, lit)):
                outs.append(ch._ARR[prec](op))
        for op in (x == lit, x != lit, x < lit, x <= lit, x > lit, x >= lit, ch.cond(x > lit, x, lit)):
            outs.append(ch._ARR[prec](op))
        return outs
    stmts, outs = record(build)
    binds = [(a.var, prec, 16, 8, 1, 0, 100 + i) for i, a in enumerate(outs[1:])]
    st, src = source(stmts, binds)
    assert st == 0, src[:3000]


def test_rng_all_variants_compile():
    def build():
        outs = []
        for variant in (ch.RNG_PHILOX, ch.RNG_THREEFRY):
            for G in (ch.RNGf32, ch.RNGf64, ch.RNGu32, ch.RNGi32):
                g = G(variant, 1)
                outs.append(ch._ARR[G.PREC](ch.rng_uniform_make(g, 12, 5)))
                outs.append(ch._ARR[G.PREC](ch.rng_uniform_make(g, 16, 5)))
                if G in (ch.RNGf32, ch.RNGf64):
                    outs.append(ch._ARR[G.PREC](ch.rng_normal_make(g, 10, 3)))
                    outs.append(ch._ARR[G.PREC](ch.rng_normal_make(g, 64, 3)))
        return outs
    stmts, outs = record(build)
    binds = [(a.var, a.prec, a.W, a.H, 1, 0, 100 + i) for i, a in enumerate(outs)]
    st, src = source(stmts, binds)
    assert st == 0, src[:3000]


def test_unsupported_opcode_is_reported():
    stmts = [(1, 1, [ch._sc(1.0), ch._op(5 + 2), ch._op(999)])]
    st, msg = source(stmts)
    assert st == -2 and "999" in msg


def test_malformed_trace_is_invalid():
    stmts = [(1, 1, [ch._op(11)])]
    st, _ = source(stmts)
    assert st == -1


def test_border_tiles_staged_by_tma_with_wrapped_patches():
    """On an image of at least one staged tile, border tiles take the same TMA
    load as interior ones (zero fill outside the image) and then replace only
    the elements outside the image by wrapped loads; StencilBorderTma=0 keeps
    the all-wrapped staging."""
    from tests.test_gpu_trace import kirsch_expr
    W = H = 512

    def build():
        A = ch._ARR[4](_raw=([ch._bc(L.BC_MEMORY, buffer=7), ch._sc(1), ch._sc(H), ch._sc(W), ch._op(66)], W, H, 1))
        return A, ch.Arrayf32(kirsch_expr(ch, A, W, H))
    stmts, (A, K) = record(build)
    st, src = source(stmts, [(K.var, 4, W, H, 1, 0, 8)])
    assert st == 0, src
    assert src.count("tma_load_3d(tile0") == 1 and "if (!interior && tile_ok)" in src
    assert "if (y >= 0 && y < H && x >= 0 && x < W) continue;" in src
    st0, src0 = source(stmts, [(K.var, 4, W, H, 1, 0, 8)], "StencilBorderTma=0")
    assert st0 == 0 and "if (!interior && tile_ok)" not in src0 and "if (interior) {" in src0
