"""BF16 tcgen05 tile GEMMs (the closure network's building block) against fp32 matmuls."""

from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k,a_mn,b_mn", [(64, 80, 0, 0), (64, 64, 1, 0), (64, 128, 0, 1),
                                           (64, 128, 1, 1), (16, 16, 0, 0), (256, 32, 0, 0),
                                           (80, 48, 1, 1)])
def test_tile_gemm_matches_fp32(n, k, a_mn, b_mn):
    import torch

    from pyspectral_b200 import _lib, build

    build.build()
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(n * 1000 + k)
    A = torch.randn(128, k, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    Ag = A.T.contiguous() if a_mn else A.contiguous()
    Bg = B.T.contiguous() if b_mn else B.contiguous()
    D = torch.full((128, n), float("nan"), device="cuda")
    st = lib.sp_mma_tile_check(ctypes.c_void_p(Ag.data_ptr()), ctypes.c_void_p(Bg.data_ptr()),
                               ctypes.c_void_p(D.data_ptr()), n, k, a_mn, b_mn,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.sp_create_error()
    torch.testing.assert_close(D, ref, rtol=1e-5, atol=1e-4)
