"""tcgen05 BF16 GEMM (corrector building block) against torch FP32 matmul.  Needs a B200.

Products of bf16 values are exact in fp32, so the only difference from the reference is the
fp32 summation order: rel-L2 <= 1e-5.
"""
import ctypes as ct

import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _gemm(A, B, N, K, Df=None, Db=None, bias=None, resid=None, preact=None, act=0, k_splits=1):
    from fvm_solver_b200 import _lib
    lib = _lib.load()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    M = A.shape[0]
    ldd = (Df if Df is not None else Db).stride(0)
    rc = lib.fvm_gemm_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K, k_splits,
                           _lib.ptr(bias), _lib.ptr(resid), resid.stride(0) if resid is not None else 0,
                           _lib.ptr(Df), _lib.ptr(Db), ldd, _lib.ptr(preact), act, err.data_ptr(), _lib.stream_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return err


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (300, 32, 128), (1000, 128, 64), (257, 256, 192), (5, 64, 128)])
def test_gemm_matches_torch(M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    D = torch.full((M, N), float("nan"), device="cuda")
    _gemm(A, B, N, K, Df=D)
    ref = A.float() @ B.float().t()
    assert rel_l2(D.cpu().numpy(), ref.cpu().numpy()) < 1e-5


def test_gemm_epilogue():
    g = torch.Generator(device="cuda").manual_seed(7)
    M, N, K = 333, 64, 128
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    resid = torch.randn(M, N, device="cuda", generator=g)
    D = torch.empty(M, N, device="cuda")
    Db = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    pre = torch.empty(M, N, device="cuda")
    _gemm(A, B, N, K, Df=D, Db=Db, bias=bias, resid=resid, preact=pre, act=1)
    z = A.float() @ B.float().t() + bias
    ref = torch.nn.functional.silu(z) + resid
    assert rel_l2(pre.cpu().numpy(), z.cpu().numpy()) < 1e-5
    assert rel_l2(D.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    assert rel_l2(Db.float().cpu().numpy(), ref.cpu().numpy()) < 1e-2


def test_gemm_split_k():
    g = torch.Generator(device="cuda").manual_seed(11)
    M, N, K = 128, 64, 64 * 40
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    D = torch.zeros(M, N, device="cuda")
    _gemm(A, B, N, K, Df=D, k_splits=8)
    ref = A.float() @ B.float().t()
    assert rel_l2(D.cpu().numpy(), ref.cpu().numpy()) < 1e-5
