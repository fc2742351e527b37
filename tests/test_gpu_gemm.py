"""tcgen05 BF16 GEMM (C = A B^T, f32 accumulate) against a PyTorch fp32 reference.

The kernel is the tensor-core building block of the learned warm start.  Its
inputs are bf16, so the reference multiplies the same bf16 values in fp32;
the only difference left is the summation order (tolerance 1e-4 relative to
the largest |C|).
"""
import pytest

pytestmark = pytest.mark.gpu


def _run(ctx, m, n, k, k_splits=1, lda=None, ldb=None, seed=0):
    import torch
    g = torch.Generator(device="cuda:0")
    g.manual_seed(seed)
    lda = lda or k
    ldb = ldb or k
    a_full = torch.randn(m, lda, device="cuda:0", generator=g).to(torch.bfloat16)
    b_full = torch.randn(n, ldb, device="cuda:0", generator=g).to(torch.bfloat16)
    c = torch.full((m, n), float("nan"), device="cuda:0")
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_gemm_bf16_nt(ctx.ptr, m, n, k, a_full.data_ptr(), lda, b_full.data_ptr(), ldb,
                                      c.data_ptr(), n, k_splits))
    ref = a_full[:, :k].float() @ b_full[:, :k].float().T
    err = (c - ref).abs().max().item()
    scale = ref.abs().max().item()
    return err, scale


@pytest.mark.parametrize("n", [16, 64, 128])
def test_gemm_square_tiles(gpu_ctx, n):
    err, scale = _run(gpu_ctx, 256, n, 128)
    assert err <= 1e-4 * scale, (err, scale)


@pytest.mark.parametrize("m,k", [(1, 64), (129, 64), (1000, 128), (4099, 192), (3, 40)])
def test_gemm_ragged_edges(gpu_ctx, m, k):
    # rows beyond m and k beyond the operand are zero-filled by the tensor maps
    ld = ((k + 7) // 8) * 8
    err, scale = _run(gpu_ctx, m, 64, k, lda=ld, ldb=ld)
    assert err <= 1e-4 * scale, (err, scale)


def test_gemm_many_tiles_persistent(gpu_ctx):
    # more 128-row tiles than SMs: every CTA loops over several tiles
    err, scale = _run(gpu_ctx, 148 * 128 * 3 + 77, 64, 128, seed=3)
    assert err <= 1e-4 * scale, (err, scale)


@pytest.mark.parametrize("splits", [2, 7, 40])
def test_gemm_split_k_weight_gradient_shape(gpu_ctx, splits):
    # tall-skinny reduction shape of a weight gradient: [128 x n] [64 x n]^T
    err, scale = _run(gpu_ctx, 128, 64, 50_000, k_splits=splits, seed=5)
    assert err <= 1e-4 * scale, (err, scale)


def test_gemm_rejects_bad_shapes(gpu_ctx):
    import torch
    from spectral_init_b200.api import InvalidArgument
    a = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda:0")
    c = torch.zeros(128, 32, device="cuda:0")
    st = gpu_ctx.lib.si_gemm_bf16_nt(gpu_ctx.ptr, 128, 32, 64, a.data_ptr(), 64, a.data_ptr(), 64,
                                     c.data_ptr(), 32, 1)
    with pytest.raises(InvalidArgument):
        gpu_ctx.check(st)
