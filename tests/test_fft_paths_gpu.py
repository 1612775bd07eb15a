"""The three FFT pass families give the same operator applies.

BDG_FFT_PATH selects the family per call: `reg` (line transforms in
registers, the default), `ct` (compile-time sized shared-memory stages) and
`generic` (runtime-sized stages).  The oracle pins the register path on a
64^3 dipolar problem; the other geometries compare the families with each
other at sizes where the oracle is slow.  Together they cover every line
length of the register kernels (16, 32, 48, 64, 96, 128, 256), 2D and 3D,
real and complex fields, FP64 and FP32, and the two-field M half (dipolar
exchange) as well as the one-field halves.  The random dipolar kernel used
here is not symmetric under k -> -k, so the test also checks that every
family treats the DC and Nyquist terms of a real row the same way.

Tolerance: 1e-12 relative (max-norm) between FP64 results; FP32 results
against the FP64 generic path to 2e-5.
"""
import numpy as np
import pytest

from oracle import bdg_oracle as O

pytestmark = pytest.mark.gpu

REL64 = 1e-12
REL32 = 2e-5


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


def _device_problem(B, dim, N, cplx, seed):
    rng = np.random.default_rng(seed)
    S = int(np.prod(N))
    H = S if cplx else (N[0] // 2 + 1) * S // N[0]
    L = [0.5 * n for n in N]
    dc = B.DeviceContext(dim, N, L, cplx)
    wf = rng.standard_normal(S) + (1j * rng.standard_normal(S) if cplx else 0.0)
    dc.set_fields(ltK=1 + rng.random(S), ltM=2 + rng.random(S), wf=wf, pK=0.5 + rng.random(S),
                  pM=0.5 + rng.random(S), mu=0.9, vdd=rng.standard_normal(H), g_ddi=0.6, dipolar=(dim == 3))
    return dc, rng, S


def _apply(torch, dc, op, prec, X, path, monkeypatch):
    monkeypatch.setenv("BDG_FFT_PATH", path)
    cplx = np.iscomplexobj(X)
    if prec:
        tdt = torch.complex64 if cplx else torch.float32
    else:
        tdt = torch.complex128 if cplx else torch.float64
    xt = torch.tensor(X).to(tdt).cuda()
    yt = torch.zeros_like(xt)
    torch.cuda.synchronize()
    dc.apply_ptr(op, prec, xt.data_ptr(), X.shape[1], yt.data_ptr(), X.shape[1], X.shape[0])
    dc.synchronize()
    return yt.cpu().numpy().astype(np.complex128 if cplx else np.float64)


GEOMS = [
    (3, [128, 32, 16], False),
    (3, [96, 48, 16], False),
    (3, [256, 16, 32], False),
    (3, [32, 64, 128], True),
    (3, [16, 16, 48], True),
    (2, [128, 96], True),
    (2, [48, 256], False),
    (2, [64, 16], False),
]


@pytest.mark.parametrize("geom", GEOMS, ids=lambda g: f"{g[0]}d-{'x'.join(map(str, g[1]))}-{'z' if g[2] else 'd'}")
def test_fft_paths_agree(geom, bdg, monkeypatch):
    torch = _torch()
    dim, N, cplx = geom
    dc, rng, S = _device_problem(bdg, dim, N, cplx, 3)
    ncol = 3
    X = rng.standard_normal((ncol, 2 * S))
    if cplx:
        X = X + 1j * rng.standard_normal((ncol, 2 * S))
    for op in (bdg.OP_LREP, bdg.OP_TLREP, bdg.OP_M, bdg.OP_K):
        Xo = X if op in (bdg.OP_LREP, bdg.OP_TLREP) else np.ascontiguousarray(X[:, :S])
        ref = _apply(torch, dc, op, 0, Xo, "generic", monkeypatch)
        for path in ("ct", "reg"):
            e = relerr(_apply(torch, dc, op, 0, Xo, path, monkeypatch), ref)
            assert e < REL64, (op, path, e)
        e32 = relerr(_apply(torch, dc, op, 1, Xo, "reg", monkeypatch), ref)
        assert e32 < REL32, (op, "reg f32", e32)


def test_register_path_against_oracle_64cubed(bdg, monkeypatch):
    """Lrep and T_Lrep of a 64^3 dipolar problem: register kernels against
    the oracle's per-column FFT restatement of the reference operators."""
    torch = _torch()
    dim, N, L = 3, [64, 64, 64], [10.0, 10.0, 10.0]
    rng = np.random.default_rng(21)
    oc = O.Ctx(dim, N, L, False)
    O.set_system(oc)
    S = oc.size
    oc.localTermK, oc.localTermM = 1.0 + rng.random(S), 2.0 + rng.random(S)
    oc.precond_sqrtK, oc.precond_sqrtM = 0.5 + rng.random(S), 0.5 + rng.random(S)
    oc.mu = 0.8
    oc.wf = rng.standard_normal(S)
    O.dipolar_set_kernel(oc, 0.7, [0.0, 0.0, 1.0], 4.0)
    oc.dipolar = True
    dc = bdg.DeviceContext(dim, N, L, False)
    dc.set_fields(ltK=oc.localTermK, ltM=oc.localTermM, wf=oc.wf, pK=oc.precond_sqrtK, pM=oc.precond_sqrtM,
                  mu=oc.mu, vdd=oc.longRngInt, g_ddi=oc.g_ddi, dipolar=True)
    X = rng.standard_normal((2, 2 * S))
    for op, ref in ((bdg.OP_LREP, O.matmulLrep), (bdg.OP_TLREP, O.precondLrep)):
        got = _apply(torch, dc, op, 0, X, "reg", monkeypatch)
        for c in range(X.shape[0]):
            e = relerr(got[c], ref(oc, X[c]))
            assert e < REL64, (op, c, e)
