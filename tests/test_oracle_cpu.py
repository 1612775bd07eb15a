"""The CPU oracle against the reference's own known answers (pins the
oracle), plus oracle self-consistency.  No GPU."""
import math

import numpy as np
import pytest

import cases
from oracle import bdg_oracle as O


@pytest.mark.parametrize("case", cases.CASES, ids=lambda f: f.__name__)
def test_known_answer_oracle(case):
    cases.check(case(cases.OracleAdapter))


def _uniform_1d(cplx):
    ctx = O.Ctx(1, [64], [2 * math.pi], cplx)
    O.set_system(ctx)
    O.set_wavefunction(ctx, np.ones(64))
    O.set_local_interactions(ctx, lambda n: n, lambda n: n)
    O.set_mu(ctx, 1.0)
    return ctx


def test_oracle_solver_1d_uniform():
    """tests/test_bdg_1d_uniform.c:60-140 restated on the oracle solver:
    two eigenvalues at sqrt(1.25), at least one at sqrt(8), within 1%."""
    ctx = _uniform_1d(False)
    X0 = O.gaussian_block_bpositive(ctx, 10, 0)
    r = O.ilobpcg(ctx, X0, 4, 200, 1e-4)
    assert r.converged >= 4
    ev = r.eigvals[:4]
    E1, E2 = math.sqrt(1.25), math.sqrt(8.0)
    assert np.sum(np.abs(ev - E1) < 0.01 * E1) == 2
    assert np.sum(np.abs(ev - E2) < 0.01 * E2) >= 1


def test_oracle_solver_d_vs_z():
    """tests/test_bdg_1d_uniform.c:142-230: complex path matches real path."""
    rd = O.ilobpcg(_uniform_1d(False), O.gaussian_block_bpositive(_uniform_1d(False), 10, 0), 4, 200, 1e-4)
    cz = _uniform_1d(True)
    rz = O.ilobpcg(cz, O.gaussian_block_bpositive(cz, 10, 0), 4, 200, 1e-4)
    E1 = math.sqrt(1.25)
    d1 = rd.eigvals[np.argmin(np.abs(rd.eigvals - E1))]
    z1 = rz.eigvals[np.argmin(np.abs(rz.eigvals - E1))]
    assert abs(d1 - z1) < 1e-4


def test_rr_pencil_properties():
    """C^T (S^T B S) C = I and C^T (S^T A S) C = diag(lam) on a random
    definite pencil."""
    rng = np.random.default_rng(0)
    S = 50
    K = rng.standard_normal((S, S)); K = K @ K.T + S * np.eye(S)
    M = rng.standard_normal((S, S)); M = M @ M.T + S * np.eye(S)
    Xu = rng.standard_normal((6, S))
    X = np.concatenate([Xu, Xu + 0.1 * rng.standard_normal((6, S))], axis=1)
    AX = np.concatenate([X[:, :S] @ K, X[:, S:] @ M], axis=1)
    Guu = X[:, :S] @ X[:, :S].T
    Gvv = X[:, S:] @ X[:, S:].T
    Guv = X[:, :S] @ X[:, S:].T
    Ga = X @ AX.T
    lam, C = O.rr_pencil(Guu, Gvv, Guv, Ga, 3)
    Gb = Guv + Guv.T
    assert np.allclose(C.T @ Gb @ C, np.eye(3), atol=1e-10)
    assert np.allclose(C.T @ Ga @ C, np.diag(lam), atol=1e-8 * np.max(np.abs(lam)))
    assert np.all(np.diff(lam) >= 0)


def test_oracle_dense_known_answer_1d():
    """Solver eigenvalues vs a dense eig(K M) of the same 1D trapped problem."""
    N, L = 48, 12.0
    ctx = O.Ctx(1, [N], [L])
    O.set_system(ctx)
    x = (np.arange(N) - N / 2) * L / N
    psi = np.exp(-x * x / 2)
    psi /= math.sqrt(np.sum(psi ** 2) * L / N)
    O.set_trap_array(ctx, 0.5 * x * x)
    O.set_wavefunction(ctx, psi)
    O.set_local_interactions(ctx, lambda n: 0.0 * n, lambda n: 0.0 * n)
    O.set_mu(ctx, 0.5)
    E = np.eye(N)
    Kd = O.matmulK(ctx, E).T
    Md = O.matmulM(ctx, E).T
    w2 = np.sort(np.linalg.eigvals(Kd @ Md).real)
    omega = np.sqrt(np.clip(w2, 0, None))
    X0 = O.gaussian_block_bpositive(ctx, 8, 3)
    r = O.ilobpcg(ctx, X0, 4, 300, 1e-10)
    assert r.converged >= 4
    assert np.allclose(r.eigvals[1:4], omega[1:4], rtol=1e-7)


def test_oracle_dense_known_answer_3d():
    """The oracle iLOBPCG on a 3D trapped dipolar problem (8^3, contact and
    dipolar terms, mu below the spectrum so K and M are positive definite)
    against the dense spectrum: omega = sqrt(eig(K M)) of the assembled
    operators, five lowest modes to 1e-11 relative."""
    N, L = [8, 8, 8], [6.0, 6.0, 6.0]
    oc0 = O.Ctx(3, N, L)
    O.set_system(oc0)
    c = O.grid_coords(oc0)
    Z, Y, X = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    psi = np.exp(-0.5 * (X ** 2 + Y ** 2 + 2 * Z ** 2)).reshape(-1)
    psi /= math.sqrt(np.sum(psi ** 2) * np.prod([l / n for l, n in zip(L, N)]))
    oc = O.build_problem(N, L, [1.0, 1.0, 1.5], 5.0, 2.0, psi, 0.2, Rc=3.0)
    E = np.eye(oc.size)
    Kd = O.matmulK(oc, E).T
    Md = O.matmulM(oc, E).T
    assert np.abs(Kd - Kd.T).max() < 1e-12 and np.abs(Md - Md.T).max() < 1e-12
    omega = np.sqrt(np.sort(np.linalg.eigvals(Kd @ Md).real)[:5])
    r = O.ilobpcg(oc, O.gaussian_block_bpositive(oc, 10, 1), 5, 400, 1e-11)
    assert r.converged >= 5
    assert np.all(np.abs(r.eigvals[:5] - omega) / omega < 1e-11), (r.eigvals[:5], omega)


def test_oracle_dense_known_answer_3d_complex():
    """The complex (_z) oracle path on the same 8^3 problem with psi0 carrying
    a global phase e^{0.3 i}: K and M are Hermitian, and the iLOBPCG modes
    equal the dense sqrt(eig(K M)) and the real problem's spectrum."""
    N, L = [8, 8, 8], [6.0, 6.0, 6.0]
    oc0 = O.Ctx(3, N, L)
    O.set_system(oc0)
    c = O.grid_coords(oc0)
    Z, Y, X = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    psi = np.exp(-0.5 * (X ** 2 + Y ** 2 + 2 * Z ** 2)).reshape(-1)
    psi /= math.sqrt(np.sum(psi ** 2) * np.prod([l / n for l, n in zip(L, N)]))
    spectra = []
    for cplx in (False, True):
        oc = O.build_problem(N, L, [1.0, 1.0, 1.5], 5.0, 2.0, psi * (np.exp(0.3j) if cplx else 1.0), 0.2, Rc=3.0,
                             complex_psi0=cplx)
        E = np.eye(oc.size, dtype=complex if cplx else float)
        Kd = O.matmulK(oc, E).T
        Md = O.matmulM(oc, E).T
        assert np.abs(Kd - Kd.conj().T).max() < 1e-12 and np.abs(Md - Md.conj().T).max() < 1e-12
        omega = np.sqrt(np.sort(np.linalg.eigvals(Kd @ Md).real)[:5])
        r = O.ilobpcg(oc, O.gaussian_block_bpositive(oc, 10, 1), 5, 400, 1e-11)
        assert r.converged >= 5
        assert np.all(np.abs(r.eigvals[:5] - omega) / omega < 1e-11)
        spectra.append(omega)
    assert np.allclose(spectra[0], spectra[1], rtol=1e-12)


def test_oracle_goldstone_deflation_complex_psi0():
    """Goldstone deflation on the complex path: the stationary 16^3 dipolar
    ground state with a global phase e^{0.3 i} as complex psi0 gives the real
    problem's four lowest nonzero modes (true residual <= 1e-8) to 1e-13."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_fixtures as FX

    fx = FX.load("gs16")
    N = [int(v) for v in fx["N"]]
    L = [float(v) for v in fx["L"]]
    om = [float(v) for v in fx["omegas"]]
    g, gdd, rc, mu = float(fx["g"]), float(fx["gdd"]), float(fx["rc"]), float(fx["mu"])
    ev = []
    for cplx in (False, True):
        psi = fx["psi"] * (np.exp(0.3j) if cplx else 1.0)
        oc = O.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc, complex_psi0=cplx)
        proj, _ = O.goldstone_projector(oc)
        r = O.ilobpcg(oc, O.gaussian_block_bpositive(oc, 8, 0), 4, 400, 1e-8, proj=proj,
                      criterion=O.CONV_TRUE_RESIDUAL)
        assert r.converged >= 4
        ev.append(r.eigvals[:4])
    assert np.all(np.abs(ev[0] - ev[1]) / ev[0] < 1e-13)


def test_oracle_p_normalisation_does_not_change_the_solve():
    """The projected P enters [X, P] without its own SVQB (the default of all
    three restatements): same eigenvalues (1e-12) and iteration count within
    one of the normalised variant on the 16^3 dipolar problem."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_fixtures as FX

    fx = FX.load("gs16")
    N = [int(v) for v in fx["N"]]
    L = [float(v) for v in fx["L"]]
    om = [float(v) for v in fx["omegas"]]
    oc = O.build_problem(N, L, om, float(fx["g"]), float(fx["gdd"]), fx["psi"], float(fx["mu"]), Rc=float(fx["rc"]))
    proj, _ = O.goldstone_projector(oc)
    X0 = O.gaussian_block_bpositive(oc, 8, 0)
    runs = [O.ilobpcg(oc, X0, 4, 400, 1e-8, proj=proj, criterion=O.CONV_TRUE_RESIDUAL, normalize_p=norm)
            for norm in (True, False)]
    assert all(r.converged >= 4 for r in runs)
    assert np.all(np.abs(runs[0].eigvals[:4] - runs[1].eigvals[:4]) / runs[0].eigvals[:4] < 1e-12)
    assert abs(runs[0].iters - runs[1].iters) <= 1, (runs[0].iters, runs[1].iters)
