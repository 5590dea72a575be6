"""The control-variate network's tensor-core kernels (tcgen05, BF16 inputs,
FP32 accumulation) against torch's FP32 products of the same BF16 values.
Tolerance: |D - D_ref| <= 1e-5 * sum_k |a_ik b_jk| (FP32 summation order)."""
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("m,n,k,batch", [(128, 128, 16, 1), (256, 128, 128, 2),
                                         (128, 16, 64, 3), (384, 128, 208, 1),
                                         (128, 16, 1024, 2)])
def test_gemm_bf16_matches_fp32_reference(cub, ctx, m, n, k, batch):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k + batch)
    a = torch.randn(batch, m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(batch, n, k, device="cuda", generator=g).to(torch.bfloat16)
    d = cub.mlp_gemm_bf16(a, b)
    ref = torch.bmm(a.float(), b.float().transpose(1, 2))
    scale = torch.bmm(a.float().abs(), b.float().abs().transpose(1, 2))
    err = (d - ref).abs()
    assert bool((err <= 1e-5 * scale + 1e-30).all()), float((err / scale).max())
