"""GPU operator parity: the CUDA library against the CPU oracle.

Every case calls the library through its C ABI (single-column host entry
points of the reference's internal API, or the block device entry points of
bdg/bdg_cuda.h) and compares with the oracle on the same seeded inputs.
Tolerance: operator applies match to 1e-12 relative (max-norm) in FP64;
FP32 applies to 2e-5 relative.
"""
import math

import numpy as np
import pytest

import cases
from oracle import bdg_oracle as O

pytestmark = pytest.mark.gpu

REL64 = 1e-12
REL32 = 2e-5


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("case", cases.CASES, ids=lambda f: f.__name__)
def test_known_answer_gpu(case, bdg):
    """The reference's own known answers on the GPU path."""
    cases.check(case(cases.GpuAdapter))


def _random_problem(dim, N, L, cplx, seed, dipolar):
    """Random smooth-ish fields on both the oracle and the library."""
    rng = np.random.default_rng(seed)
    oc = O.Ctx(dim, N, L, cplx)
    O.set_system(oc)
    size = oc.size
    ltK = 1.0 + rng.random(size)
    ltM = 2.0 + rng.random(size)
    pK = 0.5 + rng.random(size)
    pM = 0.5 + rng.random(size)
    wf = rng.standard_normal(size) + (1j * rng.standard_normal(size) if cplx else 0.0)
    oc.localTermK, oc.localTermM = ltK.copy(), ltM.copy()
    oc.precond_sqrtK, oc.precond_sqrtM = pK.copy(), pM.copy()
    oc.mu = 0.7
    oc.wf = np.asarray(wf, dtype=oc.ctype)
    import bdg_lobpcg_b200 as B

    gc = B.OperatorContext(dim, N, L, cplx)
    gc.set("localTermK", ltK)
    gc.set("localTermM", ltM)
    gc.set("precond_sqrtK", pK)
    gc.set("precond_sqrtM", pM)
    gc.set_scalar("mu", 0.7)
    gc.set("wf", wf)
    if dipolar:
        O.dipolar_set_kernel(oc, 0.8, [0.2, 0.3, 1.0], 0.4 * L[0])
        oc.dipolar = True
        gc.set_dipolar_kernel(0.8, [0.2, 0.3, 1.0], 0.4 * L[0])
        gc.set_scalar("dipolar", 1)
    return oc, gc, rng


GEOMS = [
    (1, [64], [6.0], False),
    (1, [48], [5.0], True),
    (2, [16, 12], [4.0, 3.0], False),
    (2, [12, 16], [3.0, 4.0], True),
    (3, [8, 6, 4], [2.0, 1.5, 1.0], False),
    (3, [16, 16, 16], [8.0, 8.0, 8.0], False),
    (3, [24, 20, 18], [6.0, 5.0, 4.5], True),
    (3, [32, 32, 32], [16.0, 16.0, 16.0], False),
    (3, [48, 24, 16], [12.0, 6.0, 4.0], False),
]


@pytest.mark.parametrize("geom", GEOMS, ids=lambda g: f"{g[0]}d-{'x'.join(map(str, g[1]))}-{'z' if g[3] else 'd'}")
def test_operator_parity(geom, bdg):
    dim, N, L, cplx = geom
    dip = dim == 3
    oc, gc, rng = _random_problem(dim, N, L, cplx, 11, dip)
    size = oc.size
    dt = np.complex128 if cplx else np.float64

    def rnd(n):
        v = rng.standard_normal(n)
        return (v + 1j * rng.standard_normal(n)) if cplx else v

    for name in ("kinetic", "matmulK", "matmulM", "precondK", "precondM"):
        x = rnd(size).astype(dt)
        e = relerr(gc.apply(name, x), getattr(O, name)(oc, x))
        assert e < REL64, (name, e)
    for name in ("matmulLrep", "precondLrep", "matmulSwap"):
        x = rnd(2 * size).astype(dt)
        e = relerr(gc.apply(name, x), getattr(O, name)(oc, x))
        assert e < REL64, (name, e)
    if dip:
        x = rnd(size).astype(dt)
        e = relerr(gc.apply("dipolar_conv", x), O.dipolar_conv(oc, x))
        assert e < REL64, ("dipolar_conv", e)


def test_fft_roundtrip_mixed_radix(bdg):
    """tests/test_setup.c:192-286: forward then backward returns size * x,
    including the mixed-radix 8x6x4 r2c case and a 2D c2c case."""
    import bdg_lobpcg_b200 as B

    for dim, N, L, cplx in ((3, [8, 6, 4], [1.0, 2.0, 3.0], False), (2, [16, 8], [1.0, 1.0], True),
                            (1, [32], [1.0], False)):
        c = B.OperatorContext(dim, N, L, cplx)
        size = int(np.prod(N))
        i = np.arange(size)
        x = ((i % 7) - 3.0) if not cplx else (i + 1j * (size - i)).astype(np.complex128)
        X = c.fft(True, x)
        # the forward transform matches numpy's (FFTW's) layout
        ref = np.fft.rfftn(np.asarray(x, float).reshape(N[::-1])) if not cplx else np.fft.fftn(x.reshape(N[::-1]))
        assert relerr(X, ref.reshape(-1)) < 1e-13
        y = c.fft(False, X)
        assert np.max(np.abs(y / size - x)) < 1e-10


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("prec", [0, 1])
def test_block_apply_device(cplx, prec, bdg):
    """Batched block applies on device memory (bdgd_apply) for LREP and TLREP
    on 12 columns of a 32^3 dipolar problem, FP64 and FP32."""
    torch = _torch()
    import bdg_lobpcg_b200 as B

    dim, N, L = 3, [32, 32, 32], [12.0, 12.0, 12.0]
    oc, gc, rng = _random_problem(dim, N, L, cplx, 5, True)
    size = oc.size
    dc = B.DeviceContext(dim, N, L, cplx)
    dc.set_fields(ltK=oc.localTermK, ltM=oc.localTermM, wf=oc.wf, pK=oc.precond_sqrtK, pM=oc.precond_sqrtM,
                  mu=oc.mu, vdd=oc.longRngInt, g_ddi=oc.g_ddi, dipolar=True)
    ncol = 12
    X = rng.standard_normal((ncol, 2 * size))
    if cplx:
        X = X + 1j * rng.standard_normal((ncol, 2 * size))
    if prec == 1:
        tdt = torch.complex64 if cplx else torch.float32
    else:
        tdt = torch.complex128 if cplx else torch.float64
    xt = torch.tensor(X).to(tdt).cuda()
    yt = torch.zeros_like(xt)
    for op, ref in ((B.OP_LREP, O.matmulLrep), (B.OP_TLREP, O.precondLrep)):
        torch.cuda.synchronize()
        dc.apply_ptr(op, prec, xt.data_ptr(), 2 * size, yt.data_ptr(), 2 * size, ncol)
        dc.synchronize()
        got = yt.cpu().numpy().astype(np.complex128 if cplx else np.float64)
        xin = xt.cpu().numpy().astype(np.complex128 if cplx else np.float64)
        e = relerr(got, ref(oc, xin))
        assert e < (REL32 if prec else REL64), (op, prec, e)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("prec", [0, 1])
def test_gram_blocks(cplx, prec, bdg):
    """bdgd_gram: Guu, Gvv, Guv, Ga of a tall-skinny block against numpy
    (FP64 accumulation; FP32 inputs are compared on their rounded values)."""
    torch = _torch()
    import bdg_lobpcg_b200 as B

    rng = np.random.default_rng(3)
    half, k = 5000, 70
    n = 2 * half
    S = rng.standard_normal((k, n))
    AS = rng.standard_normal((k, n))
    if cplx:
        S = S + 1j * rng.standard_normal((k, n))
        AS = AS + 1j * rng.standard_normal((k, n))
    tdt = {(0, False): torch.float64, (1, False): torch.float32, (0, True): torch.complex128,
           (1, True): torch.complex64}[(prec, cplx)]
    St = torch.tensor(S).to(tdt).cuda()
    At = torch.tensor(AS).to(tdt).cuda()
    S = St.cpu().numpy().astype(np.complex128 if cplx else np.float64)
    AS = At.cpu().numpy().astype(np.complex128 if cplx else np.float64)
    out = torch.zeros(4 * k * k * (2 if cplx else 1), dtype=torch.float64, device="cuda")
    dc = B.DeviceContext(1, [half], [1.0], cplx)
    torch.cuda.synchronize()
    dc.gram_ptr(prec, cplx, half, k, St.data_ptr(), n, At.data_ptr(), n, out.data_ptr())
    dc.synchronize()
    o = out.cpu().numpy()
    if cplx:
        o = o.view(np.complex128)
    G = o.reshape(4, k, k).transpose(0, 2, 1)  # column-major blocks
    Su, Sv = S[:, :half], S[:, half:]
    refs = [Su.conj() @ Su.T, Sv.conj() @ Sv.T, Su.conj() @ Sv.T, S.conj() @ AS.T]
    for g, r in zip(G, refs):
        assert relerr(g, r) < 1e-12


@pytest.mark.parametrize("cplx", [False, True])
def test_gram_blocks_streamk_vs_split(cplx, bdg, monkeypatch):
    """The stream-K Gram schedule (default) against numpy and against the
    row-split schedule (BDG_GRAM_SPLIT=1): k = 150 columns (three 64-wide
    tiles, sym and non-sym tasks), an odd half length (padded tile rows, tasks
    over n and over n/2 rows on one work line)."""
    torch = _torch()
    import bdg_lobpcg_b200 as B

    rng = np.random.default_rng(8)
    half, k = 40001, 150
    n = 2 * half
    S = rng.standard_normal((k, n))
    AS = rng.standard_normal((k, n))
    if cplx:
        S = S + 1j * rng.standard_normal((k, n))
        AS = AS + 1j * rng.standard_normal((k, n))
    tdt = torch.complex128 if cplx else torch.float64
    St = torch.tensor(S).to(tdt).cuda()
    At = torch.tensor(AS).to(tdt).cuda()
    dc = B.DeviceContext(1, [64], [1.0], cplx)  # the Gram does not depend on the grid
    outs = []
    for split in (False, True):
        if split:
            monkeypatch.setenv("BDG_GRAM_SPLIT", "1")
        out = torch.full((4 * k * k * (2 if cplx else 1),), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        dc.gram_ptr(0, cplx, half, k, St.data_ptr(), n, At.data_ptr(), n, out.data_ptr())
        dc.synchronize()
        o = out.cpu().numpy()
        if cplx:
            o = o.view(np.complex128)
        outs.append(o.reshape(4, k, k).transpose(0, 2, 1))
    Su, Sv = S[:, :half], S[:, half:]
    refs = [Su.conj() @ Su.T, Sv.conj() @ Sv.T, Su.conj() @ Sv.T, S.conj() @ AS.T]
    for g, g2, r in zip(outs[0], outs[1], refs):
        assert np.all(np.isfinite(g))
        assert relerr(g, r) < 1e-12
        assert relerr(g, g2) < 1e-13


def test_block_update_vs_numpy(bdg):
    """bdgd_block_update (fused FP64 DMMA basis update) against numpy: an odd
    row count under an even leading dimension (a ragged last row pair), terms
    of 64, 37 and 70 columns (partial and multiple 32-column stages), small
    matrices with leading dimensions above k and 8-byte-offset pointers, 100
    output columns (two column tiles), beta != 0 (read-modify-write), beta = 0
    over a NaN-filled output (must not be read), a term-less output (left
    untouched) and the unsupported FP32 form (status -3, nothing launched)."""
    torch = _torch()
    import bdg_lobpcg_b200 as B

    rng = np.random.default_rng(11)
    n, ld = 80001, 80002
    ks = [64, 37, 70]
    ncol = 100
    S = [torch.tensor(rng.standard_normal((k, ld))).cuda() for k in ks]  # column-major n x k (rows contiguous)
    ldcs = [k + 3 for k in ks]
    Cbuf = [torch.tensor(rng.standard_normal(1 + ldc * ncol)).cuda() for ldc in ldcs]
    Cm = [c.cpu().numpy()[1:].reshape(ncol, ldc)[:, :k] for c, ldc, k in zip(Cbuf, ldcs, ks)]
    Y0 = rng.standard_normal((ncol, ld))
    Y1 = torch.tensor(Y0).cuda()
    Y2 = torch.full((ncol, ld), float("nan"), dtype=torch.float64, device="cuda")
    Y3 = torch.tensor(Y0).cuda()
    dc = B.DeviceContext(1, [64], [1.0], False)
    terms = [(s.data_ptr(), k, c.data_ptr() + 8, ldc) for s, k, c, ldc in zip(S, ks, Cbuf, ldcs)]
    torch.cuda.synchronize()
    rc = dc.block_update(0, False, n, ld, [(Y1.data_ptr(), ncol, -0.7, 1.3, terms),
                                           (Y2.data_ptr(), ncol, 2.0, 0.0, terms[1:]),
                                           (Y3.data_ptr(), ncol, 1.0, 0.0, [(S[0].data_ptr(), 0, Cbuf[0].data_ptr(), 1)])])
    assert rc == 0
    dc.synchronize()
    Sn = [s.cpu().numpy()[:, :n] for s in S]
    ref1 = -0.7 * sum(c @ s for c, s in zip(Cm, Sn)) + 1.3 * Y0[:, :n]
    ref2 = 2.0 * sum(c @ s for c, s in zip(Cm[1:], Sn[1:]))
    y1, y2 = Y1.cpu().numpy(), Y2.cpu().numpy()
    assert relerr(y1[:, :n], ref1) < 1e-13
    assert relerr(y2[:, :n], ref2) < 1e-13
    assert np.array_equal(y1[:, n:], Y0[:, n:])  # padding rows untouched
    assert np.all(np.isnan(y2[:, n:]))
    assert np.array_equal(Y3.cpu().numpy(), Y0)
    assert dc.block_update(1, False, n, ld, [(Y1.data_ptr(), ncol, 1.0, 0.0, terms)]) == -3
    dc.close()


def test_solver_fused_update_matches_blas(bdg, monkeypatch):
    """A 32^3 FP64 solve with the fused update kernel and with cuBLAS GEMMs
    (BDG_UPDATE_BLAS=1) reaches the same eigenvalues (1e-12 relative)."""
    from bdg_lobpcg_b200 import problems

    cfg = problems.config(32)
    psi, mu, _, _, V = problems.ground_state(bdg, cfg)
    ev = []
    for blas in (False, True):
        if blas:
            monkeypatch.setenv("BDG_UPDATE_BLAS", "1")
        p, _ = problems.build(bdg, cfg, psi, mu, V, "f64")
        assert p.solve() == 0
        assert p.stats()["max_true_residual"] <= 1e-8
        ev.append(p.eigenvalues().copy())
        p.close()
    assert np.max(np.abs(ev[0] - ev[1]) / np.abs(ev[1])) < 1e-12
