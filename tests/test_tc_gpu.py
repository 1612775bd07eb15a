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


def _gram_blocks(torch, rows, k, seed, kind):
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = 2 * rows
    X = torch.randn(k, n, dtype=torch.float64, device="cuda", generator=g)
    if kind == "weighted":
        # localised columns with a wide dynamic range (like psi0-weighted
        # modes), a few tiny columns and one zero column
        r = torch.linspace(-4, 4, n, dtype=torch.float64, device="cuda")
        X = X * torch.exp(-0.5 * r * r)[None, :] * torch.logspace(0, -9, k, dtype=torch.float64, device="cuda")[:, None]
        X[k // 2] = 0.0
    AX = torch.randn(k, n, dtype=torch.float64, device="cuda", generator=g) * 1e3
    return X, AX


@pytest.mark.parametrize("rows,k,kind", [(4096, 64, "random"), (40000, 70, "weighted"), (262144, 192, "random"),
                                         (131072, 130, "weighted")])
def test_gram_tc_matches_reference(bdg, monkeypatch, rows, k, kind):
    """The tensor-core FP64 Gram (int8 digits on tcgen05, exact int32 sums)
    against the FP64 DMMA Gram and an extended-precision product: normwise
    |G - G_ref| <= 1e-14 |a_i| |b_j| (the DMMA kernel is held to the same)."""
    torch = _torch()
    X, AX = _gram_blocks(torch, rows, k, rows + k, kind)
    n = 2 * rows
    dc = bdg.DeviceContext(3, [16, 16, 16], [8.0] * 3, False)
    outs = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("BDG_GRAM_TC", mode)
        out = torch.full((4 * k * k,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        dc.gram_ptr(0, False, rows, k, X.data_ptr(), n, AX.data_ptr(), n, out.data_ptr())
        dc.synchronize()
        outs[mode] = out.cpu().numpy().reshape(4, k, k)  # column-major k x k each: [j][i]
    x = X.cpu().numpy().astype(np.longdouble)
    ax = AX.cpu().numpy().astype(np.longdouble)
    xu, xv = x[:, :rows], x[:, rows:]
    ref = [xu @ xu.T, xv @ xv.T, xu @ xv.T, x @ ax.T]  # [i][j]
    nu = np.sqrt(np.sum(xu * xu, axis=1))
    nv = np.sqrt(np.sum(xv * xv, axis=1))
    nx = np.sqrt(np.sum(x * x, axis=1))
    na = np.sqrt(np.sum(ax * ax, axis=1))
    scale = [np.outer(nu, nu), np.outer(nv, nv), np.outer(nu, nv), np.outer(nx, na)]
    for mode, o in outs.items():
        for q in range(4):
            got = o[q].T  # [i][j]
            sc = np.maximum(scale[q], 1e-300)
            err = np.abs(got.astype(np.longdouble) - ref[q]) / sc
            assert np.all(np.isfinite(got)), (mode, q)
            assert float(err.max()) < 1e-14, (mode, q, float(err.max()))
    dc.close()


@pytest.mark.parametrize("rows,k,kind", [(4096, 64, "random"), (40000, 70, "weighted"), (262144, 192, "random"),
                                         (131072, 130, "weighted")])
def test_gram_tc_fp32_matches_reference(bdg, monkeypatch, rows, k, kind):
    """The tensor-core Gram of FP32 blocks (4 int8 digits per value, the FP32
    phase of the mixed form) against the exact FP64 product of the same FP32
    values: |G - G_ref| <= 2^-30 (max|a_i| sum|b_j| + max|b_j| sum|a_i|),
    twice the bound of its 31-bit fixed-point rounding (the DMMA kernel,
    which widens the values to FP64, is held to 1e-14 of the same scale)."""
    torch = _torch()
    X, AX = _gram_blocks(torch, rows, k, rows + 3 * k, kind)
    X, AX = X.float(), AX.float()
    n = 2 * rows
    dc = bdg.DeviceContext(3, [16, 16, 16], [8.0] * 3, False)
    outs = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("BDG_GRAM_TC", mode)
        out = torch.full((4 * k * k,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        dc.gram_ptr(1, False, rows, k, X.data_ptr(), n, AX.data_ptr(), n, out.data_ptr())
        dc.synchronize()
        outs[mode] = out.cpu().numpy().reshape(4, k, k)
    x = X.cpu().numpy().astype(np.float64)
    ax = AX.cpu().numpy().astype(np.float64)
    xu, xv = x[:, :rows], x[:, rows:]
    pairs = [(xu, xu), (xv, xv), (xu, xv), (x, ax)]
    for q, (a, b) in enumerate(pairs):
        ref = a @ b.T
        ma, mb = np.abs(a).max(axis=1), np.abs(b).max(axis=1)
        sa, sb = np.abs(a).sum(axis=1), np.abs(b).sum(axis=1)
        scale = np.maximum(np.outer(ma, sb) + np.outer(sa, mb), 1e-300)
        for mode, tol in (("0", 1e-14), ("1", 2.0 ** -30)):
            got = outs[mode][q].T
            assert np.all(np.isfinite(got)), (mode, q)
            err = float((np.abs(got - ref) / scale).max())
            assert err < tol, (mode, q, err)
    dc.close()


@pytest.mark.parametrize("fixture,nev,prec", [("gs16", 4, "f64"), ("c1_32", 8, "f64"), ("c1_32", 8, "mixed")])
def test_solve_with_tc_gram_matches_dmma(bdg, monkeypatch, fixture, nev, prec):
    """The whole solve with the tensor-core Gram and update (FP64, or the
    mixed form with its FP32-phase Gram on the tensor cores): same eigenvalues
    as with the DMMA kernels (1e-12 relative) and the true residual <= tol."""
    import os

    from oracle import bdg_oracle as O

    f = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{fixture}.npz"))
    N = [int(v) for v in f["N"]]
    L = [float(v) for v in f["L"]]
    om = [float(v) for v in f["omegas"]]
    g, gdd, rc, mu, psi = float(f["g"]), float(f["gdd"]), float(f["rc"]), float(f["mu"]), f["psi"]
    m, tol = 2 * nev, 1e-8
    oc = O.Ctx(3, N, L)
    X0 = O.gaussian_block_bpositive(oc, m, 0)
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("BDG_GRAM_TC", mode)
        monkeypatch.setenv("BDG_UPDATE_TC", mode)
        p = bdg.Problem(3, N, L)
        p.set_system()
        p.set_trap(O.harmonic_trap(oc, om))
        p.set_wavefunction(psi)
        p.set_local_interactions(lambda n: g * n, lambda n: g * n)
        p.set_dipolar(gdd, [0.0, 0.0, 1.0], rc)
        p.set_mu(mu)
        p.set_solver_params(nev, m, 400, tol)
        p.set_initial_block(X0)
        p.set_goldstone_deflation(True)
        p.set_convergence(bdg.CONV_TRUE_RESIDUAL)
        p.set_precision(bdg.PREC_MIXED if prec == "mixed" else bdg.PREC_F64)
        assert p.solve() == 0 and p.converged() >= nev
        st = p.stats()
        assert st["max_true_residual"] <= tol
        res[mode] = (p.eigenvalues()[:nev].copy(), st["iterations"])
        p.close()
    e0, e1 = res["0"][0], res["1"][0]
    assert np.all(np.abs(e1 - e0) / np.abs(e0) < 1e-12), (e0, e1)
    assert abs(res["1"][1] - res["0"][1]) <= 3


@pytest.mark.parametrize("n,m,beta", [(8192, 16, 0.0), (100000, 64, 0.0), (65536, 40, 1.0)])
def test_update_tc_matches_reference(bdg, monkeypatch, n, m, beta):
    """The tensor-core FP64 basis update Y = alpha sum_b S_b C_b + beta Y
    (the iteration's X' = [X P W] Cx, P' = [P W] Cp and a beta = 1
    projection shape) against the DMMA update and an extended-precision
    product: normwise |Y - Y_ref| <= 1e-14 (|S_r| |C_c| + |beta Y|)."""
    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(n + m)
    blk = {nm: torch.randn(m, n, dtype=torch.float64, device="cuda", generator=g) for nm in ("X", "P", "W")}
    r = torch.linspace(-3, 3, n, dtype=torch.float64, device="cuda")
    blk["W"] = blk["W"] * torch.exp(-r * r)[None, :] * 1e-6  # small, localised search directions
    Cx = torch.randn(m, 3 * m, dtype=torch.float64, device="cuda", generator=g)  # (3m x m) column-major
    Cp = torch.randn(m, 2 * m, dtype=torch.float64, device="cuda", generator=g)
    Y0 = torch.randn(m, n, dtype=torch.float64, device="cuda", generator=g)
    e8 = 8

    def terms(names, Cm):
        return [(blk[nm].data_ptr(), m, Cm.data_ptr() + i * m * e8, Cm.shape[1]) for i, nm in enumerate(names)]

    results = {}
    dc = bdg.DeviceContext(3, [16, 16, 16], [8.0] * 3, False)
    for mode in ("0", "1"):
        monkeypatch.setenv("BDG_UPDATE_TC", mode)
        ys = [Y0.clone(), Y0.clone()]
        outs = [(ys[0].data_ptr(), m, 1.0, beta, terms(("X", "P", "W"), Cx)),
                (ys[1].data_ptr(), m, -1.0, beta, terms(("P", "W"), Cp))]
        torch.cuda.synchronize()
        assert dc.block_update(0, False, n, n, outs) == 0
        dc.synchronize()
        results[mode] = [y.cpu().numpy() for y in ys]
    S = {k: v.cpu().numpy().astype(np.longdouble) for k, v in blk.items()}
    cx = Cx.cpu().numpy().astype(np.longdouble)  # [col][k]
    cp = Cp.cpu().numpy().astype(np.longdouble)
    y0 = Y0.cpu().numpy().astype(np.longdouble)
    Sx = np.concatenate([S["X"], S["P"], S["W"]])  # (3m, n)
    Sp = np.concatenate([S["P"], S["W"]])
    refs = [cx @ Sx + beta * y0, -(cp @ Sp) + beta * y0]
    scales = [np.outer(np.sqrt((cx * cx).sum(1)), np.sqrt((Sx * Sx).sum(0))) + abs(beta) * np.abs(y0),
              np.outer(np.sqrt((cp * cp).sum(1)), np.sqrt((Sp * Sp).sum(0))) + abs(beta) * np.abs(y0)]
    for mode, ys in results.items():
        for q in range(2):
            err = np.abs(ys[q].astype(np.longdouble) - refs[q]) / np.maximum(scales[q], 1e-300)
            assert np.all(np.isfinite(ys[q])), (mode, q)
            assert float(err.max()) < 1e-14, (mode, q, float(err.max()))
    dc.close()
