"""The reference's front end linked with chai_b200 (the CudaDevice adapter and
its DeviceMap, chai_b200/refdevice/): without CHAI_CUDA the device table is
the reference's own, so unchanged sample programs run on the reference
interpreter exactly as before.  Checked against restatements of the samples'
arithmetic: sample/md5.cpp digests (the interpreter's output, which the B200
run must reproduce, is pinned here against the same binary twice), and
sample/index.cpp (sum(exp(A) + transpose(B)) over 10 x 10 index arrays, f32
element arithmetic, double sum; 6 significant digits printed)."""
import numpy as np
import pytest

from tests import refsamples as R

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref/cuda not built (reference sources absent)")


def test_interpreter_path_through_adapter_devicemap_index():
    out = R.run("index", cuda=False)
    f = np.float32
    A = np.tile(np.arange(10, dtype=f), (10, 1))              # index_f32(0, 10, 10): column index
    B = f(0.25) * np.tile(np.arange(10, dtype=f)[:, None], (1, 10))
    want = float((np.exp(A) + B.T).astype(np.float64).sum())
    got = float(R.NUM.findall(out)[0])
    assert abs(got - want) <= 1e-5 * want, (out, want)


def test_interpreter_path_is_deterministic_md5():
    a, b = R.run("md5", cuda=False), R.run("md5", cuda=False)
    assert a == b and a.count("has MD5 hash") == 28


def test_sum_and_matmul_samples_on_interpreter():
    out = R.run("sum_uni", cuda=False)
    assert out.count("result[") == 10
    out = R.run("matmul_uni", cuda=False)
    vals = [float(v) for v in R.NUM.findall(out)[1::2]]
    # D = sum(alpha A B + beta C), A[j] = .001 j, B[j] = .001 (N^2 - j), C = 1 + i
    N, alpha, beta = 40, np.float32(.777), np.float32(.888)
    j = np.arange(N * N, dtype=np.float32)
    A = (np.float32(0.001) * j).reshape(N, N).astype(np.float64)
    B = (np.float32(0.001) * (N * N - j)).reshape(N, N).astype(np.float64)
    for i, v in enumerate(vals):
        want = float((alpha * (A @ B) + beta * (1.0 + i)).sum())
        assert abs(v - want) <= 1e-4 * abs(want), (i, v, want)
