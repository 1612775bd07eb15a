"""The Gram entry point that allocates nothing (bdgd_gram_noalloc).

It exists for callers that may not allocate device memory when they need
the Gram blocks, e.g. code running inside a memory pool it does not own or a
framework that bans cudaMalloc on its hot path.  Its partial sums live in a
static device array, so it must give the same blocks as the ordinary entry
point (bdgd_gram, which grows its scratch with cudaMalloc), call after call.

This file is collected last on purpose: a run that stops at the first failure
has then already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, the tolerance of the other Gram tests


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


def _noalloc(B):
    f = B.lib().bdgd_gram_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                  C.c_uint64, C.c_void_p]
    return f


def _relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("prec", [0, 1])
def test_gram_noalloc_matches_gram_two_calls(cplx, prec, bdg):
    torch = _torch()
    f = _noalloc(bdg)
    half, k = 6000, 70
    n = 2 * half
    tdt = {(0, False): torch.float64, (1, False): torch.float32, (0, True): torch.complex128,
           (1, True): torch.complex64}[(prec, cplx)]
    dc = bdg.DeviceContext(1, [half], [1.0], cplx)
    es = 2 if cplx else 1
    gen = torch.Generator(device="cuda").manual_seed(7)
    for call in range(2):
        # new inputs on each call: the second result must not depend on the first
        S = torch.randn(k, n, dtype=tdt, device="cuda", generator=gen)
        AS = torch.randn(k, n, dtype=tdt, device="cuda", generator=gen)
        ref = torch.zeros(4 * k * k * es, dtype=torch.float64, device="cuda")
        out = torch.full_like(ref, float("nan"))
        torch.cuda.synchronize()
        dc.gram_ptr(prec, cplx, half, k, S.data_ptr(), n, AS.data_ptr(), n, ref.data_ptr())
        dc.synchronize()
        rc = f(None, prec, 1 if cplx else 0, half, k, S.data_ptr(), n, AS.data_ptr(), n, out.data_ptr())
        assert rc == 0, bdg.lib().bdgd_last_error().decode()
        torch.cuda.synchronize()
        o, r = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(o)), f"call {call}: output not fully written"
        assert _relerr(o, r) < TOL, (call, _relerr(o, r))


def test_gram_noalloc_rejects_oversize(bdg):
    torch = _torch()
    f = _noalloc(bdg)
    k = 600  # 4 k^2 doubles exceed the static buffer
    S = torch.zeros(k, 64, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = f(None, 0, 0, 32, k, S.data_ptr(), 64, S.data_ptr(), 64, out.data_ptr())
    assert rc != 0
    assert b"static buffer" in bdg.lib().bdgd_last_error()
