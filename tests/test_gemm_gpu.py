"""The surrogate's BF16 tensor-core GEMM (tcgen05.mma with TMEM accumulators),
through the C ABI, against a PyTorch fp32 product of the same bf16 inputs.
Tolerance: 1e-4 relative to the row scale (fp32 accumulation in a different
order; inputs identical)."""
import numpy as np
import pytest

import sysmat_b200

pytestmark = pytest.mark.gpu


def _ref(a, b):
    return a.float() @ b.float().T


@pytest.mark.parametrize("m,n,k,n_tile", [(128, 256, 64, 256), (300, 200, 96, 256), (2048, 256, 256, 256),
                                          (256, 64, 2048, 64), (64, 128, 16, 128), (129, 257, 130, 256)])
def test_gemm_matches_fp32_reference(m, n, k, n_tile):
    import torch
    torch.manual_seed(m + n + k)
    a = torch.randn(m, k, device="cuda").bfloat16()
    b = torch.randn(n, k, device="cuda").bfloat16()
    c = torch.full((m, n), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    sysmat_b200.gemm_bf16(m, n, k, a.data_ptr(), (k, 1), b.data_ptr(), (k, 1), c.data_ptr(), n, n_tile=n_tile,
                          error=err.data_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = _ref(a, b)
    scale = ref.abs().amax(1, keepdim=True).clamp_min(1e-6)
    assert ((c - ref).abs() / scale).max().item() <= 1e-4


def test_gemm_strided_operands_scale_bias_accumulate():
    import torch
    torch.manual_seed(3)
    m, n, k = 200, 128, 300
    at = torch.randn(k, m, device="cuda").bfloat16()          # A stored transposed: A[i][k] = at[k][i]
    bt = torch.randn(k, n, device="cuda").bfloat16()          # B[j][k] = bt[k][j]
    rs = torch.rand(m, device="cuda") + 0.5
    bias = torch.randn(n, device="cuda")
    c0 = torch.randn(m, n, device="cuda")
    c = c0.clone()
    sysmat_b200.gemm_bf16(m, n, k, at.data_ptr(), (1, m), bt.data_ptr(), (1, n), c.data_ptr(), n,
                          row_scale=rs.data_ptr(), bias=bias.data_ptr(), accumulate=True, n_tile=128)
    torch.cuda.synchronize()
    ref = rs[:, None] * (at.float().T @ bt.float()) + bias[None, :] + c0
    scale = ref.abs().amax(1, keepdim=True)
    assert ((c - ref).abs() / scale).max().item() <= 1e-4
