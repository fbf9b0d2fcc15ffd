"""Inline OpenCL kernels (ProgramCL) beyond the scalar language, on the GPU:
vector arithmetic with swizzles and literals, comparisons / select /
conversions with saturation and rounding modes, double vectors with as_type,
the integer built-ins, local and global atomics, work-group copies into
__local vectors, and image2d_t parameters read and written through samplers.
Expected values are numpy in the same arithmetic (bit-exact), except the
bilinear sampler (1e-6)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
f32, f64, u32, i32 = np.float32, np.float64, np.uint32, np.int32


@pytest.fixture
def ch(chai_dev):
    import chai_b200.api as ch
    return ch


SWZ = """
__kernel void swz(__global const float* a, __global float* out)
{
    const size_t i = get_global_id(0);
    float4 v = vload4(i, a);
    float4 u = v * (float4)(1.0f, 2.0f, 3.0f, 4.0f) + (float4)(0.5f);
    u.xy = u.yx;
    u.zw += (float2)(1.0f, -1.0f);
    u.s0 = u.s3 * 2.0f;
    float8 r = (float8)(u, u.wzyx);
    r.odd = r.even - 1.0f;
    vstore8(r, i, out);
}
"""


def test_vector_arithmetic_swizzles_and_literals(ch):
    n4 = 256
    a = np.random.default_rng(1).uniform(-4, 4, 4 * n4).astype(f32)
    A = ch.make1(a)
    out = ch.Arrayf32(ch.zeros_f32(8 * n4))
    ch.ProgramCL(SWZ)("swz", A, out)(n4, 64)
    got = out.read1().reshape(n4, 8)
    u = a.reshape(n4, 4) * np.array([1, 2, 3, 4], f32) + f32(0.5)
    u[:, [0, 1]] = u[:, [1, 0]]
    u[:, 2] = u[:, 2] + f32(1)
    u[:, 3] = u[:, 3] + f32(-1)
    u[:, 0] = u[:, 3] * f32(2)
    r = np.concatenate([u, u[:, ::-1]], axis=1)
    r[:, 1::2] = r[:, 0::2] - f32(1)
    assert np.array_equal(got, r)


CMPSEL = """
__kernel void cmpsel(__global const float* a, __global const float* b, __global float* out, __global int* iout)
{
    const size_t i = get_global_id(0);
    float4 x = vload4(i, a), y = vload4(i, b);
    int4 c = x > y;
    vstore4(select(x, y, c), i, out);
    vstore4(convert_int4_rtn(x * 100.0f), 3 * i, iout);
    vstore4(convert_int4_sat(y * 3.0e9f), 3 * i + 1, iout);
    vstore4(c + (int4)(any(c), all(c), any(c == 0), all(c == 0)), 3 * i + 2, iout);
}
"""


def test_compare_select_and_conversions(ch):
    n4 = 128
    rng = np.random.default_rng(2)
    a = rng.uniform(-1, 1, 4 * n4).astype(f32)
    b = rng.uniform(-1, 1, 4 * n4).astype(f32)
    b[:8] = a[:8] - f32(0.5)          # a row where every x > y
    out = ch.Arrayf32(ch.zeros_f32(4 * n4))
    iout = ch.Arrayi32(ch.zeros_i32(12 * n4))
    ch.ProgramCL(CMPSEL)("cmpsel", ch.make1(a), ch.make1(b), out, iout)(n4, 32)
    x, y = a.reshape(n4, 4), b.reshape(n4, 4)
    c = np.where(x > y, -1, 0).astype(i32)
    assert np.array_equal(out.read1().reshape(n4, 4), np.where(c < 0, y, x))
    got = iout.read1().reshape(n4, 3, 4)
    assert np.array_equal(got[:, 0], np.floor(x * f32(100)).astype(i32))
    sat = np.clip(np.trunc((y * f32(3.0e9)).astype(f64)), -2.0 ** 31, 2.0 ** 31 - 1).astype(i32)
    assert np.array_equal(got[:, 1], sat)
    flags = np.stack([(c < 0).any(1), (c < 0).all(1), (c == 0).any(1), (c == 0).all(1)], 1).astype(i32)
    assert np.array_equal(got[:, 2], c + flags)
    assert got[0, 2, 1] == -1 + 1       # all(c) on the row with every x > y


DVEC = """
#pragma OPENCL EXTENSION cl_khr_fp64 : enable
__kernel void dv(__global const double* a, __global double* out, __global long* bits)
{
    const size_t i = get_global_id(0);
    double2 v = vload2(i, a);
    long2 l = convert_long2_rte(v * 1.0e6);
    vstore2(v * v + convert_double2(l), i, out);
    bits[i] = as_long(v.x) ^ l.y;
}
"""


def test_double_vectors_long_conversion_and_as_type(ch):
    n2 = 256
    a = np.random.default_rng(3).uniform(-50, 50, 2 * n2)
    out = ch.Arrayf64(ch.zeros_f64(2 * n2))
    bits = ch.Arrayf64(ch.zeros_f64(n2))           # written as 64-bit integers
    ch.ProgramCL(DVEC)("dv", ch.make1(a), out, bits)(n2, 64)
    v = a.reshape(n2, 2)
    ll = np.rint(v * 1.0e6).astype(np.int64)
    assert np.array_equal(out.read1().reshape(n2, 2), v * v + ll.astype(f64))
    assert np.array_equal(bits.read1().view(np.int64), v[:, 0].view(np.int64) ^ ll[:, 1])


INTS = """
__kernel void ints(__global const uint* a, __global const uint* b, __global uint* out)
{
    const size_t i = get_global_id(0);
    uint4 x = vload4(i, a), y = vload4(i, b);
    vstore4(rotate(x, y), 5 * i, out);
    vstore4(clz(x), 5 * i + 1, out);
    vstore4(popcount(x), 5 * i + 2, out);
    vstore4(add_sat(x, y), 5 * i + 3, out);
    vstore4(mul_hi(x, y), 5 * i + 4, out);
}
"""


def test_integer_builtins_on_vectors(ch):
    n4 = 64
    rng = np.random.default_rng(4)
    a = rng.integers(0, 2 ** 32, 4 * n4, dtype=np.uint64).astype(u32)
    b = rng.integers(0, 2 ** 32, 4 * n4, dtype=np.uint64).astype(u32)
    a[:4] = [0, 1, 0x80000000, 0xFFFFFFFF]
    b[:4] = [0, 32, 31, 0xFFFFFFFF]
    out = ch.Arrayu32(ch.zeros_u32(20 * n4))
    ch.ProgramCL(INTS)("ints", ch.make1(a), ch.make1(b), out)(n4, 32)
    got = out.read1().reshape(n4, 5, 4)
    x, y = a.astype(np.uint64).reshape(n4, 4), b.astype(np.uint64).reshape(n4, 4)
    s = y & np.uint64(31)
    rot = ((x << s) | (x >> (np.uint64(32) - s))) & np.uint64(0xFFFFFFFF)
    clz = np.array([32 - int(v).bit_length() for v in x.ravel()]).reshape(n4, 4)
    pop = np.array([bin(int(v)).count("1") for v in x.ravel()]).reshape(n4, 4)
    sat = np.minimum(x + y, np.uint64(0xFFFFFFFF))
    hi = (x * y) >> np.uint64(32)
    for k, want in enumerate((rot, clz, pop, sat, hi)):
        assert np.array_equal(got[:, k].astype(np.uint64), want.astype(np.uint64)), k


HIST = """
__kernel void hist(__global const uint* x, __global uint* h, __local uint* lh, uint n, uint bins)
{
    const uint l = get_local_id(0);
    for (uint b = l; b < bins; b += get_local_size(0)) lh[b] = 0;
    barrier(CLK_LOCAL_MEM_FENCE);
    const size_t g = get_global_id(0);
    if (g < n) atomic_inc(&lh[x[g] % bins]);
    barrier(CLK_LOCAL_MEM_FENCE);
    for (uint b = l; b < bins; b += get_local_size(0)) atomic_add(&h[b], lh[b]);
}
__kernel void atoms(__global int* a, __global ulong* b, __global float* f)
{
    atomic_max(&a[0], (int)get_global_id(0));
    atomic_min(&a[1], -(int)get_global_id(0));
    atomic_cmpxchg(&a[2], 0, 1);
    atomic_xchg(&a[3], 7);
    atomic_or(&a[4], 1 << (get_global_id(0) & 31));
    atom_add(&b[0], (ulong)get_global_id(0));
    atomic_add(&f[0], 1.0f);
    atomic_sub(&a[5], 2);
    atomic_dec(&a[6]);
}
"""


def test_local_and_global_atomics(ch):
    n, bins = 5000, 64
    x = np.random.default_rng(5).integers(0, 2 ** 32, n, dtype=np.uint64).astype(u32)
    prog = ch.ProgramCL(HIST)
    h = ch.Arrayu32(ch.zeros_u32(bins))
    prog("hist", ch.make1(x), h, bins, u32(n), u32(bins))(5120, 256)
    assert np.array_equal(h.read1(), np.bincount(x % bins, minlength=bins).astype(u32))
    N = 1024
    a = ch.Arrayi32(ch.zeros_i32(8))
    b = ch.Arrayf64(ch.zeros_f64(1))
    f = ch.Arrayf32(ch.zeros_f32(1))
    prog("atoms", a, b, f)(N, 128)
    assert a.read1().tolist() == [N - 1, -(N - 1), 1, 7, -1, -2 * N, -N, 0]
    assert b.read1().view(np.uint64)[0] == N * (N - 1) // 2
    assert f.read1()[0] == N


TILE = """
__kernel void tile_rev(__global const float4* src, __global float4* dst, __local float4* t)
{
    event_t e = async_work_group_copy(t, src + get_group_id(0) * get_local_size(0), get_local_size(0), 0);
    wait_group_events(1, &e);
    const uint l = get_local_id(0);
    dst[get_global_id(0)] = t[get_local_size(0) - 1 - l].wzyx;
}
"""


def test_work_group_copy_into_local_vectors(ch):
    n, wg = 512, 64
    s = np.arange(4 * n, dtype=f32)
    d = ch.Arrayf32(ch.zeros_f32(4 * n))
    ch.ProgramCL(TILE)("tile_rev", ch.make1(s), d, wg)(n, wg)
    want = s.reshape(n // wg, wg, 4)[:, ::-1, ::-1].ravel()
    assert np.array_equal(d.read1(), want)


IMAGES = """
__constant sampler_t smp = CLK_NORMALIZED_COORDS_FALSE | CLK_ADDRESS_CLAMP | CLK_FILTER_NEAREST;
const sampler_t lin = CLK_NORMALIZED_COORDS_TRUE | CLK_ADDRESS_REPEAT | CLK_FILTER_LINEAR;
__kernel void nbr(__read_only image2d_t src, __write_only image2d_t dst)
{
    const int x = get_global_id(0), y = get_global_id(1);
    float4 p = read_imagef(src, smp, (int2)(x - 1, y)) + read_imagef(src, smp, (int2)(x + 1, y + 1));
    write_imagef(dst, (int2)(x, y), p);
}
__kernel void bil(__read_only image2d_t src, __global float* out, float ox, float oy)
{
    const int x = get_global_id(0), y = get_global_id(1);
    const float2 uv = (float2)(((float)x + ox) / (float)get_image_width(src),
                               ((float)y + oy) / (float)get_image_height(src));
    vstore4(read_imagef(src, lin, uv), y * get_image_width(src) + x, out);
}
__kernel void dimg(read_only image2d_t src, __global double* out)
{
    const int x = get_global_id(0), y = get_global_id(1);
    double2 v = as_double2(read_imageui(src, smp, (int2)(x, y)));
    vstore2(v * 2.0, y * get_image_width(src) + x, out);
}
"""


def _bilinear_repeat(T, s, t):
    """OpenCL 1.2 section 8.2 linear filtering with CLK_ADDRESS_REPEAT on
    normalized coordinates, in float32."""
    h, w = T.shape[:2]
    u = (s - np.floor(s)) * f32(w)
    v = (t - np.floor(t)) * f32(h)
    uu, vv = u - f32(0.5), v - f32(0.5)
    i0, j0 = int(np.floor(uu)), int(np.floor(vv))
    i1, j1 = i0 + 1, j0 + 1
    a, b = uu - np.floor(uu), vv - np.floor(vv)
    i0 += w if i0 < 0 else 0
    i1 -= w if i1 > w - 1 else 0
    j0 += h if j0 < 0 else 0
    j1 -= h if j1 > h - 1 else 0
    one = f32(1)
    return ((one - a) * (one - b)) * T[j0, i0] + (a * (one - b)) * T[j0, i1] + ((one - a) * b) * T[j1, i0] + \
        (a * b) * T[j1, i1]


def test_image_reads_writes_and_samplers(ch):
    iw, ih = 8, 6
    src = np.random.default_rng(6).uniform(-1, 1, (ih, 4 * iw)).astype(f32)
    prog = ch.ProgramCL(IMAGES)
    S = ch.make2(src)
    dst = ch.Arrayf32(ch.zeros_f32(4 * iw, ih))
    prog("nbr", S, dst)(iw, ih, 8, 2)
    T = src.reshape(ih, iw, 4)
    want = np.zeros_like(T)
    for y in range(ih):
        for x in range(iw):
            left = T[y, x - 1] if x >= 1 else np.zeros(4, f32)
            right = T[y + 1, x + 1] if (x + 1 < iw and y + 1 < ih) else np.zeros(4, f32)
            want[y, x] = left + right
    assert np.array_equal(dst.read2().reshape(ih, iw, 4), want)

    ox, oy = f32(0.3), f32(-0.7)
    out = ch.Arrayf32(ch.zeros_f32(4 * iw * ih))
    prog("bil", S, out, ox, oy)(iw, ih, 8, 2)
    got = out.read1().reshape(ih, iw, 4)
    for y in range(ih):
        for x in range(iw):
            s = (f32(x) + ox) / f32(iw)
            t = (f32(y) + oy) / f32(ih)
            np.testing.assert_allclose(got[y, x], _bilinear_repeat(T, s, t), rtol=1e-6, atol=1e-6)

    d = np.random.default_rng(7).uniform(-1, 1, (4, 2 * iw))
    dout = ch.Arrayf64(ch.zeros_f64(2 * iw * 4))
    prog("dimg", ch.make2(d), dout)(iw, 4, 8, 2)
    assert np.array_equal(dout.read1(), d.ravel() * 2.0)


HALF = """
__kernel void halves(__global const float* x, __global half* hn, __global half* hz, __global float* back)
{
    const size_t i = get_global_id(0);
    vstore_half(x[i], i, hn);
    vstore_half_rtz(x[i], i, hz);
    back[i] = vload_half(i, hn);
}
__kernel void halves4(__global const float* x, __global half* h, __global float* back)
{
    const size_t i = get_global_id(0);
    vstore_half4_rtp(vload4(i, x), i, h);
    vstore4(vload_half4(i, h), i, back);
}
"""


def _half_toward(x, direction):
    """binary16 nearest to x in the given direction (0: toward zero, +1: up)."""
    h = x.astype(np.float16)
    hf = h.astype(f32)
    if direction == 0:
        fix = np.abs(hf) > np.abs(x)
        h[fix] = np.nextafter(h[fix], np.float16(0))
    else:
        fix = hf < x
        h[fix] = np.nextafter(h[fix], np.float16(np.inf))
    return h


def test_half_storage_round_trips(ch):
    n = 256
    rng = np.random.default_rng(8)
    x = (rng.uniform(-1, 1, n) * np.logspace(-7, 4.7, n)).astype(f32)      # half subnormals .. 5e4
    x[:4] = [0.0, -0.0, 1.0 / 3.0, 65504.0]
    prog = ch.ProgramCL(HALF)
    X = ch.make1(x)
    hn, hz = ch.Arrayu32(ch.zeros_u32(n // 2)), ch.Arrayu32(ch.zeros_u32(n // 2))
    back = ch.Arrayf32(ch.zeros_f32(n))
    prog("halves", X, hn, hz, back)(n, 64)
    got_n = hn.read1().view(np.uint16).view(np.float16)
    got_z = hz.read1().view(np.uint16).view(np.float16)
    assert np.array_equal(got_n.view(np.uint16), x.astype(np.float16).view(np.uint16))
    assert np.array_equal(got_z.view(np.uint16), _half_toward(x, 0).view(np.uint16))
    assert np.array_equal(back.read1(), x.astype(np.float16).astype(f32))
    h4 = ch.Arrayu32(ch.zeros_u32(n // 2))
    back4 = ch.Arrayf32(ch.zeros_f32(n))
    prog("halves4", X, h4, back4)(n // 4, 32)
    want_p = _half_toward(x, 1)
    assert np.array_equal(h4.read1().view(np.uint16), want_p.view(np.uint16))
    assert np.array_equal(back4.read1(), want_p.astype(f32))
