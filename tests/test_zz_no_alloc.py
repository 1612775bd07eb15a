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


def _numpy_blocks(S, AS, half, cplx):
    """Guu, Gvv, Guv, Ga of the row-major (k x n) inputs in FP64 / complex128,
    as the (4, k, k) array of the column-major output blocks."""
    Su, Sv = S[:, :half], S[:, half:]
    return np.stack([Su.conj() @ Su.T, Sv.conj() @ Sv.T, Su.conj() @ Sv.T, S.conj() @ AS.T])


def _as_blocks(out, k, cplx):
    o = out.cpu().numpy()
    if cplx:
        o = o.view(np.complex128)
    return o.reshape(4, k, k).transpose(0, 2, 1)


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
        # and directly against numpy on the (rounded) inputs
        wide = np.complex128 if cplx else np.float64
        npref = _numpy_blocks(S.cpu().numpy().astype(wide), AS.cpu().numpy().astype(wide), half, cplx)
        got = _as_blocks(out, k, cplx)
        for b in range(4):
            assert _relerr(got[b], npref[b]) < TOL, (call, b, _relerr(got[b], npref[b]))


@pytest.mark.parametrize("k,cplx", [(512, False), (362, True)])
def test_gram_noalloc_at_the_size_limit(k, cplx, bdg):
    """The largest k whose 4 k^2 partial sums fit the 8 MiB static array
    (k = 512 real: exactly 2^20 doubles; k = 362 complex): one row split,
    the partials fill (almost) the whole array."""
    torch = _torch()
    f = _noalloc(bdg)
    half = 1536
    n = 2 * half
    tdt = torch.complex128 if cplx else torch.float64
    gen = torch.Generator(device="cuda").manual_seed(11)
    S = torch.randn(k, n, dtype=tdt, device="cuda", generator=gen)
    AS = torch.randn(k, n, dtype=tdt, device="cuda", generator=gen)
    out = torch.full((4 * k * k * (2 if cplx else 1),), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = f(None, 0, 1 if cplx else 0, half, k, S.data_ptr(), n, AS.data_ptr(), n, out.data_ptr())
    assert rc == 0, bdg.lib().bdgd_last_error().decode()
    torch.cuda.synchronize()
    got = _as_blocks(out, k, cplx)
    assert np.all(np.isfinite(got)), "output not fully written"
    ref = _numpy_blocks(S.cpu().numpy(), AS.cpu().numpy(), half, cplx)
    for b in range(4):
        assert _relerr(got[b], ref[b]) < TOL, (b, _relerr(got[b], ref[b]))


@pytest.mark.parametrize("k,cplx", [(600, False), (513, False), (363, True)])
def test_gram_noalloc_rejects_oversize(k, cplx, bdg):
    """One column above the limit (4 k^2 doubles, 8 k^2 for complex, above
    2^20) is refused before any launch, with the output left untouched."""
    torch = _torch()
    f = _noalloc(bdg)
    tdt = torch.complex128 if cplx else torch.float64
    S = torch.zeros(k, 64, dtype=tdt, device="cuda")
    out = torch.full((4,), 3.0, dtype=torch.float64, device="cuda")
    rc = f(None, 0, 1 if cplx else 0, 32, k, S.data_ptr(), 64, S.data_ptr(), 64, out.data_ptr())
    assert rc != 0
    assert b"static buffer" in bdg.lib().bdgd_last_error()
    torch.cuda.synchronize()
    assert torch.all(out == 3.0)
