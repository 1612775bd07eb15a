"""Tensor-core (tcgen05, sm_100a) building blocks against exact integer
arithmetic (GPU).

bdgd_tc_i8_gemm: D = A B^T with int8 operands and int32 accumulation in
tensor memory -- the MMA, shared-memory descriptors and TMEM loads that the
FP64 emulation is made of.  Integer results must match exactly.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("M,N,K", [(128, 64, 32), (256, 128, 96), (384, 192, 512)])
def test_i8_gemm_exact(bdg, M, N, K):
    torch = _torch()
    L = bdg.lib()
    f = L.bdgd_tc_i8_gemm
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                  C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p]
    rng = np.random.default_rng(M + N + K)
    a = rng.integers(-128, 128, size=(M, K), dtype=np.int8)
    b = rng.integers(-128, 128, size=(N, K), dtype=np.int8)
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda()
    D = torch.full((M, N), -7, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = f(C.c_void_p(torch.cuda.current_stream().cuda_stream), C.c_void_p(A.data_ptr()), K,
           C.c_void_p(B.data_ptr()), K, C.c_void_p(D.data_ptr()), N, M, N, K, C.c_void_p(err.data_ptr()))
    assert rc == 0, L.bdgd_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = a.astype(np.int64) @ b.astype(np.int64).T
    assert np.array_equal(D.cpu().numpy().astype(np.int64), ref)
