"""Randomised element-wise traces through the fused kernel (R5): programs
of 14 operations over three input arrays and literals, drawn from the
operations whose IEEE results are fully specified -- add, sub, mul, div,
sqrt, abs, negation, copysign (sign taken from an input, never from a NaN),
the reference's max / min (a < b ? b : a),
greater-than and cond -- evaluated by the CUDA path and by numpy with one
rounding per operation (the traced operations round one at a time; the
trace kernels are compiled without FMA contraction).  Results must be
bit-identical (NaN equal to NaN) in f32 and f64, on a shape whose size is a
multiple of 4 (128-bit loads) and a ragged one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _program(rng, nops=14):
    """[(op, operand indices)] over nodes 0..2 (the inputs), each op adding a node."""
    ops = []
    n = 3
    choices = ["add", "sub", "mul", "div", "sqrt", "abs", "neg", "copysign", "max", "min", "gt", "cond", "lit"]
    for _ in range(nops):
        op = choices[rng.integers(len(choices))]
        pick = lambda: int(n - 1 - min(rng.geometric(0.35) - 1, n - 1))     # favour recent nodes
        if op in ("sqrt", "abs", "neg"):
            ops.append((op, (pick(),)))
        elif op == "cond":
            ops.append((op, (pick(), pick(), pick())))
        elif op == "lit":
            ops.append((op, (pick(), float(rng.choice([0.5, -3.0, 1e-3, 7.25, 0.0])), int(rng.integers(4)))))
        elif op == "copysign":
            # the sign comes from an input (never NaN): the sign bit of a NaN is
            # not specified by IEEE and differs between the GPU and x86
            ops.append((op, (pick(), int(rng.integers(3)))))
        else:
            ops.append((op, (pick(), pick())))
        n += 1
    return ops


def _run(ch, ops, ins, dt):
    """Evaluate the program both ways; returns (gpu result, numpy result)."""
    import chai_b200.api as api
    ex = [api.make2(x) for x in ins]
    nv = list(ins)
    lit = lambda v: dt(v)
    with np.errstate(all="ignore"):
        for op, a in ops:
            if op == "lit":
                i, v, kind = a
                x, y = ex[i], nv[i]
                # literal on either side of add / mul / sub / div
                e, r = [(x + lit(v), y + lit(v)), (lit(v) * x, lit(v) * y), (lit(v) - x, lit(v) - y),
                        (x / lit(v), y / lit(v))][kind]
            elif op in ("sqrt", "abs", "neg"):
                x, y = ex[a[0]], nv[a[0]]
                e, r = {"sqrt": (api.sqrt(x), np.sqrt(y)), "abs": (api.abs(x), np.abs(y)),
                        "neg": (-x, -y)}[op]
            elif op == "cond":
                p, x, z = a
                e = api.cond(ex[p], ex[x], ex[z])
                r = np.where(nv[p] != 0, nv[x], nv[z])
            else:
                x, y = ex[a[0]], ex[a[1]]
                u, w = nv[a[0]], nv[a[1]]
                e, r = {"add": (x + y, u + w), "sub": (x - y, u - w), "mul": (x * y, u * w), "div": (x / y, u / w),
                        "copysign": (api.copysign(x, y), np.copysign(u, w)),
                        "max": (api.max(x, y), np.where(u < w, w, u)), "min": (api.min(x, y), np.where(u < w, u, w)),
                        "gt": (x > y, (u > w).astype(dt))}[op]
            ex.append(e)
            nv.append(np.asarray(r, dtype=dt))
    arr = api.Arrayf32(ex[-1]) if dt == np.float32 else api.Arrayf64(ex[-1])
    return arr.read2(), nv[-1]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(96, 130), (11, 37)])
def test_random_elementwise_traces_bit_exact(chai_dev, dt, shape):
    import chai_b200.api as ch
    H, W = shape
    for seed in range(10):
        rng = np.random.default_rng(1000 * seed + W)
        ins = [rng.uniform(-2.0, 2.0, (H, W)).astype(dt) for _ in range(3)]
        ins[2][rng.random((H, W)) < 0.1] = 0.0          # zeros: cond, division, copysign, signed zero
        ops = _program(rng)
        got, want = _run(ch, ops, ins, dt)
        assert got.dtype == dt and got.shape == (H, W)
        assert np.array_equal(got, want, equal_nan=True), (seed, ops)


def _int_program(rng, nops=14):
    ops = []
    n = 3
    choices = ["add", "sub", "mul", "xor", "and", "or", "shl", "shr", "max", "min", "gt"]
    for _ in range(nops):
        pick = lambda: int(n - 1 - min(rng.geometric(0.35) - 1, n - 1))
        ops.append((choices[rng.integers(len(choices))], (pick(), pick())))
        n += 1
    return ops


def _run_int(ops, ins, dt):
    import chai_b200.api as api
    ex = [api.make2(x) for x in ins]
    nv = list(ins)
    with np.errstate(all="ignore"):
        for op, (i, j) in ops:
            x, y, u, w = ex[i], ex[j], nv[i], nv[j]
            s = (w & dt(31)).astype(dt)             # shift counts are taken modulo 32
            e, r = {"add": (x + y, u + w), "sub": (x - y, u - w), "mul": (x * y, u * w), "xor": (x ^ y, u ^ w),
                    "and": (x & y, u & w), "or": (x | y, u | w), "shl": (x << y, u << s), "shr": (x >> y, u >> s),
                    "max": (api.max(x, y), np.where(u < w, w, u)), "min": (api.min(x, y), np.where(u < w, u, w)),
                    "gt": (x > y, (u > w).astype(dt))}[op]
            ex.append(e)
            nv.append(np.asarray(r, dtype=dt))
    arr = api.Arrayu32(ex[-1]) if dt == np.uint32 else api.Arrayi32(ex[-1])
    return arr.read2(), nv[-1]


@pytest.mark.parametrize("dt", [np.uint32, np.int32])
def test_random_integer_traces_bit_exact(chai_dev, dt):
    """u32 / i32 programs: add, sub, mul wrap modulo 2^32; shifts use the
    count modulo 32 (arithmetic right shift for i32); max / min / greater-than
    compare as the type does."""
    H, W = 40, 52
    info = np.iinfo(dt)
    for seed in range(8):
        rng = np.random.default_rng(77 + seed)
        ins = [rng.integers(info.min, info.max, (H, W), dtype=dt, endpoint=True) for _ in range(3)]
        ins[1][:, :4] = rng.integers(0, 40, (H, 4)).astype(dt)      # small shift counts too
        ops = _int_program(rng)
        got, want = _run_int(ops, ins, dt)
        assert got.dtype == dt and np.array_equal(got, want), (seed, ops)


@pytest.mark.parametrize("shape", [(70, 200), (33, 129), (300, 1024), (8, 12)])
def test_random_stencil_traces_bit_exact(chai_dev, shape):
    """Random constant-offset stencils: sums, differences and products of
    gather2_floor(A, X + dx, Y + dy) with |dx|, |dy| <= 4 (the 2-D tiled path:
    TMA-staged interior tiles, wrapped border tiles, shared row windows),
    against numpy's periodic roll with the same per-operation rounding."""
    import chai_b200.api as ch
    f32 = np.float32
    H, W = shape
    for seed in range(5):
        rng = np.random.default_rng(500 + 7 * seed + W)
        img = rng.standard_normal((H, W)).astype(f32)
        A = ch.make2(img)
        X, Y = ch.index_f32(0, W, H), ch.index_f32(1, W, H)
        roll = lambda dx, dy: np.roll(np.roll(img, -dy, axis=0), -dx, axis=1)
        e, r = None, None
        for _ in range(int(rng.integers(3, 9))):
            dx, dy = (int(v) for v in rng.integers(-4, 5, 2))
            g = ch.gather2_floor(A, X + f32(dx), Y + f32(dy))
            gv = roll(dx, dy)
            k = f32(rng.choice([1.0, 2.0, -0.5, 3.0]))
            if e is None:
                e, r = g * k, gv * k
                continue
            op = int(rng.integers(3))
            e, r = [(e + g * k, r + gv * k), (e - g, r - gv), (e * g, r * gv)][op]
        got = ch.Arrayf32(e).read2()
        assert np.array_equal(got, r), (seed, shape)
