"""Pins of the oracle (oracle/) against the reference itself, on the CPU.

Two sources, both produced by the reference's own code:
  * the golden fixtures in tests/golden/ (written by tests/golden/make_golden.py
    from the reference's generated Random123 text, the vendored upstream
    Random123 text and the reference's bytecode interpreter), checked always;
  * oracle/_ref (the same reference code built from its sources by
    oracle/build_ref.py), checked live on fresh seeded inputs when present.

Bars: bit-exact for generator outputs, uniforms (u32 / i32 / f32 / f64) and
for every array op whose reference accumulates in double (matmul and
matrix-vector: f32 products summed in double; sum, mean, dot_product) and for
the gather stencil; normals within 2e-6
relative (f32: the JIT text takes the logarithm and square root in float and
the sine in double, the oracle all in double) and 1e-15 (f64)."""
import ctypes as C
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLD = Path(__file__).resolve().parent / "golden"
REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"
BIJ = {"philox2x32": oracle.philox2x32, "philox4x32": oracle.philox4x32, "philox2x64": oracle.philox2x64,
       "threefry2x32": oracle.threefry2x32, "threefry2x64": oracle.threefry2x64,
       "threefry4x32": oracle.threefry4x32_chai}
PREC = {"0": oracle.U32, "1": oracle.I32, "4": oracle.F32, "8": oracle.F64}


def _gold(name):
    return np.load(GOLD / name)


# ---------------------------------------------------------------- Random123

@pytest.mark.parametrize("name", sorted(BIJ))
def test_bijection_matches_reference_jit_text(name):
    g = _gold("r123_bijections.npz")
    ctr, key, want = g[name + "_ctr"], g[name + "_key"], g[name + "_jit"]
    for i in range(ctr.shape[0]):
        np.testing.assert_array_equal(BIJ[name](ctr[i], key[i]), want[i])


@pytest.mark.parametrize("name", ["philox2x32", "philox4x32", "philox2x64", "threefry2x32", "threefry2x64"])
def test_jit_text_matches_upstream_random123(name):
    g = _gold("r123_bijections.npz")
    np.testing.assert_array_equal(g[name + "_jit"], g[name + "_up"])


def test_jit_threefry4x32_differs_from_upstream_and_oracle_follows_jit():
    """The reference JIT prints Threefry4x32 with its own lane pairing; the
    oracle (and the CUDA generator) follow the JIT text, not upstream."""
    g = _gold("r123_bijections.npz")
    assert not np.array_equal(g["threefry4x32_jit"], g["threefry4x32_up"])
    ctr, key = g["threefry4x32_ctr"], g["threefry4x32_key"]
    for i in range(ctr.shape[0]):
        np.testing.assert_array_equal(oracle.threefry4x32(ctr[i], key[i]), g["threefry4x32_up"][i])


def _wrapper_cases():
    g = _gold("r123_wrappers.npz")
    return sorted(k for k in g.files if k not in ("tid", "idx") and not k.endswith("_8_4"))


def _oracle_wrapper(name, tid, idx):
    variant, dist, prec, lanes = name.split("_")
    return oracle.rng_fill(int(lanes), variant=oracle.PHILOX if variant == "philox" else oracle.THREEFRY,
                           prec=PREC[prec], vec_len=int(lanes), dist=1 if dist == "normal" else 0, seed=int(idx),
                           first_vec=int(tid))


def _check_wrapper(name, got, want):
    if name.split("_")[1] == "uniform":
        np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    else:
        rtol = 2e-6 if want.dtype == np.float32 else 1e-15
        np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol)


@pytest.mark.parametrize("name", _wrapper_cases())
def test_rng_wrapper_matches_reference_jit_text(name):
    """Every chai uniform / normal wrapper the reference JIT prints (key and
    counter layout, int -> float conversion, Box-Muller with its 3.14159),
    at seeded and edge (vector index, seed) pairs.  The 4-lane f64 wrappers
    are not listed: f64 arrays draw 2 (or 1) values per generator call."""
    g = _gold("r123_wrappers.npz")
    for i, (tid, idx) in enumerate(zip(g["tid"], g["idx"])):
        _check_wrapper(name, _oracle_wrapper(name, tid, idx), g[name][i])


@pytest.mark.skipif(not (REF / "libr123_wrappers.so").exists(), reason="oracle/_ref not built here")
def test_rng_wrappers_live_against_reference_text():
    lib = C.CDLL(str(REF / "libr123_wrappers.so"))
    rng = np.random.default_rng(99)
    for name in _wrapper_cases():
        lanes = int(name.split("_")[3])
        dt = {"0": np.uint32, "1": np.int32, "4": np.float32, "8": np.float64}[name.split("_")[2]]
        f = getattr(lib, "w_" + name)
        f.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p]
        for tid, idx in rng.integers(0, 2 ** 32, (16, 2)):
            want = np.zeros(lanes, dtype=dt)
            f(int(tid), int(idx), want.ctypes.data)
            _check_wrapper(name, _oracle_wrapper(name, tid, idx), want)


def test_rng_fill_is_the_wrapper_sequence():
    """An array fill is wrapper(vector index, seed) for consecutive vector
    indices, lanes in order, ragged tail cut."""
    g = _gold("r123_wrappers.npz")
    n = 4 * 5 + 3
    arr = oracle.rng_fill(n, seed=42, first_vec=0)
    per = np.concatenate([_oracle_wrapper("philox_uniform_4_4", t, 42) for t in range(6)])[:n]
    np.testing.assert_array_equal(arr, per)
    row = [i for i, (t, s) in enumerate(zip(g["tid"], g["idx"])) if (t, s) == (2, 42)]
    assert row and np.array_equal(g["philox_uniform_4_4"][row[0]], arr[8:12])


# ---------------------------------------------------------------- interpreter

def interp_view(a: np.ndarray) -> np.ndarray:
    """What the reference interpreter computes on for a make2'd array: make2
    copies the rows into storage padded to a multiple of 4 elements (32-bit) or
    2 (64-bit) with zeros (memmgr/MemInterpAlloc.cpp:71-75, 152-176;
    misc/PrecType.cpp:120-132), while the interpreter's ops index that storage
    with the unpadded width (interp/BaseInterp.cpp:20-23).  For aligned widths
    this is the array itself; otherwise row y starts y * (padded - W)
    elements late.  The oracle and the CUDA path use the array as given."""
    H, W = a.shape
    vec = 2 if a.dtype == np.float64 else 4
    P = W if W % vec == 0 else vec * (1 + W // vec)
    padded = np.zeros((H, P), dtype=a.dtype)
    padded[:, :W] = a
    return padded.ravel()[:W * H].reshape(H, W)


def test_small_matmul_trace_matches_interpreter():
    """C = matmul(A, B), s = sum(C * C) at 512 x 512 (inputs: counter-layout
    Philox uniforms in [-1, 1))."""
    g = _gold("interp.npz")
    n = 512
    A = oracle.rng_fill(n * n, layout=oracle.LAYOUT_COUNTER, seed=0, limits=(-1.0, 1.0)).reshape(n, n)
    B = oracle.rng_fill(n * n, layout=oracle.LAYOUT_COUNTER, seed=1, limits=(-1.0, 1.0)).reshape(n, n)
    np.testing.assert_array_equal(A[:2], g["mm512_A_head"])
    np.testing.assert_array_equal(B[:2], g["mm512_B_head"])
    Cm = oracle.matmul_ref(A, B)
    sel = g["mm512_sel"]
    np.testing.assert_array_equal(Cm[sel[:, 0], sel[:, 1]], g["mm512_C_sel"])
    np.testing.assert_array_equal(Cm.astype(np.float64).sum(axis=1), g["mm512_rowsum"])
    s = np.float32(oracle.sum_f32(Cm * Cm))
    assert s == g["mm512_s"]


def test_ragged_gemm_matches_interpreter():
    g = _gold("interp.npz")
    C32 = oracle.matmul_ref(interp_view(g["gemm_f32_A"]), interp_view(g["gemm_f32_B"]))
    np.testing.assert_array_equal(C32, g["gemm_f32_C"])
    A, B = interp_view(g["gemm_f64_A"]), interp_view(g["gemm_f64_B"])
    C64 = np.zeros((A.shape[0], B.shape[1]))
    for k in range(A.shape[1]):          # k-ascending double accumulation
        C64 += np.outer(A[:, k], B[k])
    np.testing.assert_array_equal(C64, g["gemm_f64_C"])


def test_gemv_matches_interpreter():
    g = _gold("interp.npz")
    np.testing.assert_array_equal(oracle.matvec_ref(interp_view(g["gemv_f32_A"]), g["gemv_f32_x"]), g["gemv_f32_y"])
    np.testing.assert_array_equal(oracle.gemv_f64(interp_view(g["gemv_f64_A"]), g["gemv_f64_x"]), g["gemv_f64_y"])


def test_kirsch_gather_stencil_matches_interpreter():
    g = _gold("interp.npz")
    assert g["kirsch_img"].shape[1] % 4 == 0
    np.testing.assert_array_equal(oracle.kirsch(g["kirsch_img"]), g["kirsch_out"])


def test_interp_view_is_identity_for_aligned_widths():
    a = np.arange(24, dtype=np.float32).reshape(3, 8)
    np.testing.assert_array_equal(interp_view(a), a)
    b = np.arange(6, dtype=np.float32).reshape(2, 3)
    np.testing.assert_array_equal(interp_view(b), [[0, 1, 2], [0, 3, 4]])


def test_reductions_match_interpreter():
    g = _gold("interp.npz")
    a, b = g["reduce_a"], g["reduce_b"]
    s = oracle.sum_f32(a)
    want = g["reduce_sum_mean_dot"]
    assert np.float32(s) == want[0]
    assert np.float32(s / a.size) == want[1]
    assert np.float32(oracle.dot_f32(a, b)) == want[2]


def test_mc_payoff_matches_interpreter():
    g = _gold("interp.npz")
    Z = g["mc_Z"]
    f32 = np.float32
    S = f32(100) * np.exp(f32(0.05 - 0.5 * 0.2 * 0.2) + f32(0.2) * Z)
    payoff = np.maximum(S - f32(100), f32(0)).astype(np.float64).mean()
    assert abs(payoff - float(g["mc_payoff"])) <= 2e-6 * abs(payoff)


@pytest.mark.skipif(not (REF / "ref_driver").exists(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("shape", [(1, 1, 1), (64, 33, 17), (130, 70, 300), (96, 64, 128)])
def test_gemm_live_against_interpreter(shape):
    M, N, K = shape
    rng = np.random.default_rng(M + N + K)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    with tempfile.TemporaryDirectory() as td:
        A.tofile(td + "/A")
        B.tofile(td + "/B")
        subprocess.run([str(REF / "ref_driver"), "gemm_f32", str(M), str(N), str(K), td + "/A", td + "/B",
                        td + "/C"], check=True, capture_output=True)
        want = np.fromfile(td + "/C", dtype=np.float32).reshape(M, N)
    np.testing.assert_array_equal(oracle.matmul_ref(interp_view(A), interp_view(B)), want)
    if K % 4 == 0 and N % 4 == 0:
        np.testing.assert_array_equal(oracle.matmul_ref(A, B), want)


@pytest.mark.skipif(not (REF / "ref_driver").exists(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("W,H", [(1, 1), (3, 2), (17, 9), (8, 5)])
def test_kirsch_live_against_interpreter(W, H):
    img = np.random.default_rng(W * H).uniform(0, 1, (H, W)).astype(np.float32)
    with tempfile.TemporaryDirectory() as td:
        img.tofile(td + "/img")
        subprocess.run([str(REF / "ref_driver"), "kirsch", str(W), str(H), td + "/img", td + "/out"], check=True,
                       capture_output=True)
        want = np.fromfile(td + "/out", dtype=np.float32).reshape(H, W)
    np.testing.assert_array_equal(oracle.kirsch(interp_view(img)), want)
