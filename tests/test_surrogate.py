"""The surrogate's BF16 tensor-core GEMM against an FP32 product of the same
BF16 operands."""

import numpy as np
import pytest

from conftest import rel_l2


def _gemm(a, b, check=True):
    import torch
    from maomi_b200 import _lib
    m, k = a.shape
    n = b.shape[0]
    d = torch.full((m, n), float("nan"), dtype=torch.float32, device=a.device)
    err = torch.zeros(1, dtype=torch.int32, device=a.device)
    _lib.check(_lib.load().mm_gemm_bf16_tn(a.data_ptr(), b.data_ptr(), d.data_ptr(), m, n, k, err.data_ptr(),
                                           int(check), _lib.stream_of(a.device)), "gemm")
    return d


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(128, 32, 64), (300, 256, 4096), (576, 32, 4096), (4096, 32, 576),
                                   (200, 16, 32), (130, 96, 80)])
def test_gemm_bf16_matches_fp32_product(m, n, k):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n + k)
    a = torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((n, k), generator=g, device="cuda").to(torch.bfloat16)
    d = _gemm(a, b)
    ref = a.double() @ b.double().T
    assert torch.isfinite(d).all()
    assert rel_l2(d.cpu().numpy(), ref.cpu().numpy()) < 1e-6
