"""The surrogate's tensor-core GEMM (tcgen05.mma, TMEM accumulator, TMA-fed, 128-byte swizzled
K-major tiles) against an FP64 product of the same BF16 values: FP32 accumulation, so the error
stays at FP32 rounding of the partial sums."""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _bf16(shape, gen, scale=1.0):
    return (torch.randn(*shape, generator=gen) * scale).to(torch.bfloat16)


# split-K kernel shapes, then the persistent kernel (N in {128, 256}, K in {64, 128, 256}) with
# fewer tiles than SMs and with several tiles per CTA (ring wrap-around, both accumulators)
@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (256, 128, 320), (384, 256, 1024), (128, 256, 64),
                                   (128 * 37, 256, 256), (128 * 400, 256, 256), (128 * 1000, 128, 128),
                                   (128 * 311, 256, 64), (128 * 297, 128, 256)])
def test_gemm_store_matches_fp64(ctx, icp, m, n, k):
    gen = torch.Generator().manual_seed(m * 7 + n + k)
    a, b = _bf16((m, k), gen), _bf16((n, k), gen)
    ref = a.double().numpy() @ b.double().numpy().T
    da, db = a.cuda(), b.cuda()
    dc = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    icp.mlp_gemm_bf16(ctx, da.data_ptr(), db.data_ptr(), m, n, k, dc.data_ptr())
    got = dc.cpu().double().numpy()
    assert np.isfinite(got).all()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= 1e-5, err


@pytest.mark.parametrize("split", [1, 3, 16])
def test_gemm_split_k_accumulates(ctx, icp, split):
    m, n, k = 256, 256, 4096
    gen = torch.Generator().manual_seed(split)
    a, b = _bf16((m, k), gen, 0.1), _bf16((n, k), gen, 0.1)
    base = torch.randn(m, n, generator=gen)
    ref = base.double().numpy() + a.double().numpy() @ b.double().numpy().T
    dc = base.cuda()
    da, db = a.cuda(), b.cuda()
    torch.cuda.synchronize()
    icp.mlp_gemm_bf16(ctx, da.data_ptr(), db.data_ptr(), m, n, k, dc.data_ptr(), accumulate=True, split_k=split)
    got = dc.cpu().double().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() <= 2e-5


def test_gemm_rejects_bad_shapes(ctx, icp):
    d = torch.zeros(256, 256, dtype=torch.bfloat16, device="cuda")
    c = torch.zeros(256, 256, dtype=torch.float32, device="cuda")
    for m, n, k in [(100, 64, 64), (128, 96, 64), (128, 64, 100)]:
        with pytest.raises(icp.InvalidArgument):
            icp.mlp_gemm_bf16(ctx, d.data_ptr(), d.data_ptr(), m, n, k, c.data_ptr())


def test_pipeline_wait_that_runs_out_reports_timeout(ctx, icp):
    """The split-K GEMM's producer waits limited to one try (icp_context_set_wait_limit) give up
    while the TMA loads of a 128-chunk K range are still landing: the call returns
    ICP_ERR_TIMEOUT (the kernel drains the loads in flight with the default limit and frees its
    tensor memory before it returns), and the same context then computes the product correctly
    with the default limit."""
    import ctypes as C

    m, n, k = 256, 256, 8192
    gen = torch.Generator().manual_seed(99)
    a, b = _bf16((m, k), gen, 0.1), _bf16((n, k), gen, 0.1)
    ref = a.double().numpy() @ b.double().numpy().T
    da, db = a.cuda(), b.cuda()
    dc = torch.zeros((m, n), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    codes = []
    icp.check(icp.LIB.icp_context_set_wait_limit(ctx.handle, 1))
    try:
        for _ in range(3):
            codes.append(icp.LIB.icp_mlp_gemm_bf16(ctx.handle, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), m,
                                                   n, k, 1, C.c_void_p(dc.data_ptr()), 1))
    finally:
        icp.check(icp.LIB.icp_context_set_wait_limit(ctx.handle, 0))
    assert icp.ICP_ERR_TIMEOUT in codes and set(codes) <= {icp.ICP_OK, icp.ICP_ERR_TIMEOUT}, codes
    dc.zero_()
    torch.cuda.synchronize()
    icp.mlp_gemm_bf16(ctx, da.data_ptr(), db.data_ptr(), m, n, k, dc.data_ptr(), accumulate=True)
    got = dc.cpu().double().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() <= 2e-5
