"""chai_cuda_gemm_host: the GEMM with A, B, C in host memory, streamed through
the GPU in row blocks (copies overlapped with the GEMMs).  Its C must equal,
bit for bit, uploading the operands and calling chai_cuda_gemm on device
buffers: ragged last blocks, leading dimensions wider than the rows, alpha
and beta (C read from host memory), FP32 CUDA-core and bf16x3 tensor-core
arithmetic, and two calls in a row reusing the context's buffers."""
import ctypes as C

import numpy as np
import pytest

from chai_b200 import _lib as L

pytestmark = pytest.mark.gpu


def device_gemm(dev, A, B, C0, prec, alpha, beta):
    import torch
    M, K = A.shape
    N = B.shape[1]
    a, b = torch.from_numpy(np.ascontiguousarray(A)).cuda(), torch.from_numpy(np.ascontiguousarray(B)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(C0)).cuda()
    d = L.chai_gemm_desc(prec, 0, 0, 0, M, N, K, a.data_ptr(), K, b.data_ptr(), N, c.data_ptr(), N, alpha, beta,
                         1, 0, 0, 0)
    L.check(L.lib().chai_cuda_gemm(dev.ctx, C.byref(d)), dev.ctx)
    L.check(L.lib().chai_cuda_synchronize(dev.ctx), dev.ctx)
    return c.cpu().numpy()


def host_gemm(dev, A, B, C0, prec, alpha, beta, block_rows, pad=0):
    """Operands in (pinned) host memory with row pitches `pad` wider."""
    import torch
    M, K = A.shape
    N = B.shape[1]
    pin = lambda x, w: torch.zeros((x.shape[0], x.shape[1] + w), dtype=torch.float32).pin_memory()
    Ah, Bh, Ch = pin(A, pad), pin(B, pad), pin(C0, pad)
    Ah[:, :K] = torch.from_numpy(A)
    Bh[:, :N] = torch.from_numpy(B)
    Ch[:, :N] = torch.from_numpy(C0)
    d = L.chai_gemm_desc(prec, 0, 0, 0, M, N, K, Ah.data_ptr(), K + pad, Bh.data_ptr(), N + pad, Ch.data_ptr(),
                         N + pad, alpha, beta, 1, 0, 0, 0)
    L.check(L.lib().chai_cuda_gemm_host(dev.ctx, C.byref(d), block_rows), dev.ctx)
    return Ch[:, :N].numpy().copy()


@pytest.mark.parametrize("prec", [L.GEMM_FP32, L.GEMM_TF32, L.GEMM_BF16X3, L.GEMM_BF16X6])
@pytest.mark.parametrize("shape,block_rows,pad,beta", [((1000, 384, 200), 256, 0, 0.0),
                                                         ((700, 260, 96), 128, 4, -2.0),
                                                         ((2048, 512, 512), 0, 0, 0.0),
                                                         ((100, 64, 40), 0, 8, 0.5)])
def test_streamed_host_gemm_equals_device_gemm(chai_dev, prec, shape, block_rows, pad, beta):
    M, N, K = shape
    rng = np.random.default_rng(M + N + K)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (M, N)).astype(np.float32)
    want = device_gemm(chai_dev, A, B, C0, prec, 0.75, beta)
    for _ in range(2):
        got = host_gemm(chai_dev, A, B, C0, prec, 0.75, beta, block_rows, pad)
        assert np.array_equal(got, want)


def test_host_gemm_rejects_what_it_does_not_stream(chai_dev):
    d = L.chai_gemm_desc(L.GEMM_FP32, 1, 0, 0, 8, 8, 8, 1, 8, 1, 8, 1, 8, 1.0, 0.0, 1, 0, 0, 0)
    assert L.lib().chai_cuda_gemm_host(chai_dev.ctx, C.byref(d), 0) == -2      # CHAI_ERR_UNSUPPORTED
