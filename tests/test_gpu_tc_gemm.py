"""The tcgen05 BF16 GEMM (ostc_tc_gemm_bf16) against an FP32 product of the
same BF16 operands.  Tolerance: 1e-5 of the row scale (FP32 accumulation in a
different order)."""
import pytest

import openstc_b200 as ostc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def gemm(a, b, splits=1):
    m, k = a.shape
    n = b.shape[0]
    d = torch.zeros((splits, m, n), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = ostc.library()
    rc = lib.ostc_tc_gemm_bf16(a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0), d.data_ptr(), n, m, n, k, splits,
                               err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.ostc_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return d.sum(0)


@pytest.mark.parametrize("m,n,k,splits", [(128, 256, 256, 1), (256, 16, 256, 1), (384, 256, 16, 1),
                                          (128, 48, 64, 1), (256, 256, 4096, 8), (200, 100, 80, 1)])
def test_tc_gemm_matches_fp32(m, n, k, splits):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    d = gemm(a, b, splits)
    ref = a.float() @ b.float().T
    scale = ref.abs().amax(dim=1, keepdim=True).clamp_min(1.0)
    assert torch.all((d - ref).abs() <= 1e-5 * scale * k ** 0.5), float(((d - ref).abs() / scale).max())


def test_tc_gemm_twice_same_result():
    g = torch.Generator(device="cuda").manual_seed(1)
    a = torch.randn(256, 256, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(256, 256, device="cuda", generator=g).to(torch.bfloat16)
    assert torch.equal(gemm(a, b), gemm(a, b))
