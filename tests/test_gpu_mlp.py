"""The tensor-core tile product under the warm-start network (tcgen05, BF16 operands from
shared memory, FP32 accumulation in tensor memory), against a float64 product of the same
BF16-rounded operands: K-major operands (the forward and input-gradient products) and
MN-major operands (the weight-gradient products, which read activation tiles transposed)."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _selftest(gsb, K, N, mode, seed):
    import torch

    lib = gsb.load_library()
    g = torch.Generator().manual_seed(seed)
    if mode == 0:
        A = torch.randn(128, K, generator=g).to(torch.bfloat16)
        B = torch.randn(N, K, generator=g).to(torch.bfloat16)
        ref = A.double() @ B.double().T
    else:
        A = torch.randn(K, 128, generator=g).to(torch.bfloat16)   # A^T
        B = torch.randn(K, N, generator=g).to(torch.bfloat16)     # B^T
        ref = A.double().T @ B.double()
    Ad, Bd = A.cuda().contiguous(), B.cuda().contiguous()
    D = torch.empty(128, N, dtype=torch.float32, device="cuda")
    rc = lib.gsb_umma_selftest(ctypes.c_void_p(Ad.data_ptr()), ctypes.c_void_p(Bd.data_ptr()),
                               ctypes.c_void_p(D.data_ptr()), K, N, mode,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    return D.double().cpu().numpy(), ref.numpy()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("K,N", [(16, 16), (128, 128), (128, 16), (64, 256), (32, 48)])
def test_umma_tile_product(gsb, K, N, mode):
    d, ref = _selftest(gsb, K, N, mode, seed=K * 1000 + N + mode)
    err = np.abs(d - ref).max() / max(1.0, np.abs(ref).max())
    assert err < 1e-5, err
