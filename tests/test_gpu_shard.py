"""Sharding helpers on the GPU with one rank: a row shard of an image plus
its periodic halo through the Kirsch trace, and the row-sharded GEMM through
chai_cuda_gemm.  The exchanges themselves run as gloo ranks in
test_shard_cpu.py (every GPU run of this build has one GPU)."""
import numpy as np
import pytest

import oracle
from chai_b200 import _lib as L
from chai_b200 import shard
from tests.test_gpu_trace import kirsch_expr

pytestmark = pytest.mark.gpu


def test_kirsch_on_a_halo_slab_equals_the_whole_image(chai_dev):
    import torch

    import chai_b200.api as ch
    H, W = 120, 256
    img = oracle.rng_fill(W * H, seed=5).reshape(H, W)
    slab = shard.stencil_slab(torch.from_numpy(img).cuda(), 1)
    assert slab.shape == (H + 2, W) and slab.is_cuda
    s = slab.cpu().numpy()
    out = ch.Arrayf32(kirsch_expr(ch, ch.make2(s), W, H + 2)).read2()
    assert np.array_equal(shard.crop(torch.from_numpy(out), 1).numpy(), oracle.kirsch(img))


@pytest.mark.parametrize("rows", [(0, 300), (77, 301), (0, 0)])
def test_row_sharded_gemm_is_the_matching_rows_of_the_full_gemm(chai_dev, rows):
    import torch
    M, K, N = 301, 256, 192
    g = torch.Generator().manual_seed(3)
    A = (torch.rand((M, K), generator=g) * 2 - 1).cuda()
    B = (torch.rand((K, N), generator=g) * 2 - 1).cuda()
    r0, r1 = rows
    part = shard.gemm_rows(A[r0:r1], B, N, ctx=chai_dev.ctx, precision=L.GEMM_FP32)
    full = shard.gemm_rows(A, B, N, ctx=chai_dev.ctx, precision=L.GEMM_FP32)
    torch.cuda.synchronize()
    assert part.shape == (r1 - r0, N)
    # the FP32 CUDA-core GEMM computes each row of C from that row of A only
    assert torch.equal(part, full[r0:r1])
    ref = A.double() @ B.double()
    assert float((full.double() - ref).abs().max()) <= 2.0 ** -18 * float((A.abs().double() @ B.abs().double()).max())
