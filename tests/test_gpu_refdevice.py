"""Unchanged reference sample programs on the B200: the reference's own front
end (api/, bytecode/, common/, runtime/Scheduler) linked with chai_b200
through the CudaDevice adapter (chai_b200/refdevice/), selected by CHAI_CUDA.

Each sample binary is the reference's sample/*.cpp compiled as it is.  Its
output on the B200 must match:
  - the same binary on the reference's interpreter device, for every sample
    the interpreter runs: same text, numbers within 1e-4 relative (the
    interpreter accumulates matmul products in double, the tensor cores in
    FP32 with split bf16 operands; transcendental functions differ in the last
    ulp); integers and MD5 digests exactly;
  - for the inline-OpenCL samples (the interpreter has no ProgramCL): the
    sample's arithmetic restated -- inline_cl.cpp (f32), bitonic.cpp (the
    glibc random() stream sorted, exact), american_option_batch.cpp (20
    binomial trees in double); the printed 6 significant digits must match;
  - pi.cpp (chai Philox, which the interpreter does not implement): the oracle's
    Philox stream, exact."""
import numpy as np
import pytest

from tests import refsamples as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref/cuda not built (reference sources absent)")]


@pytest.mark.parametrize("sample", R.INTERP_SAMPLES)
def test_sample_on_b200_matches_interpreter(chai_dev, sample):
    gpu = R.run(sample, cuda=True)
    cpu = R.run(sample, cuda=False)
    assert R.same_output(gpu, cpu), (sample, gpu[:1500], cpu[:1500])


def test_inline_cl_sample(chai_dev):
    out = R.run("inline_cl", cuda=True)
    got = [float(v) for v in R.NUM.findall(out)[1::2]]
    want = R.expect_inline_cl()
    # printed with 6 significant digits
    assert len(got) == len(want) and all(abs(g - w) <= 5e-6 * abs(w) for g, w in zip(got, want)), out


def test_bitonic_sample(chai_dev):
    out = R.run("bitonic", cuda=True)
    got = [int(v) for v in R.NUM.findall(out)]
    want = sorted(R.glibc_random(16))
    assert got[1::2] == want, out


def test_american_option_batch_sample(chai_dev):
    out = R.run("american_option_batch", cuda=True)
    got = [float(v) for v in __import__("re").findall(r"is \$([-+0-9.eE]+)", out)]
    want = R.expect_american_batch()
    assert len(got) == len(want), out
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-5 * abs(w) + 1e-9, (g, w)


def test_pi_sample(chai_dev):
    import oracle
    out = R.run("pi", cuda=True)
    got = float(R.NUM.findall(out)[0])
    NSET = 1000000
    f32 = np.float32
    x = oracle.rng_fill(NSET, seed=271828, limits=(0.0, 1.0))
    y = oracle.rng_fill(NSET, seed=271828 + NSET, limits=(0.0, 1.0))
    count = f32(np.count_nonzero(np.sqrt(x * x + y * y) <= f32(1.0)))
    want = float(f32(f32(4.0) * count) / f32(NSET))
    assert abs(got - want) <= 5e-7, (out, want)
