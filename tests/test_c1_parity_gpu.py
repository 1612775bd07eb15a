"""The benchmark's CPU-runnable configuration (C1) solved on the GPU and by
the CPU oracle from the same psi0, seed and initial block.

32^3 grid over [-8, 8)^3, trap (1, 1, 2), g = 1000, eps_dd = 0.5 (dipoles
along z, cutoff 8), psi0 the committed stationary ground state
(tests/golden/c1_32.npz), nev 8, sizeSub 16, tol 1e-8 on the true residual
||K M v - w^2 v|| / ||v||, Goldstone chain deflated, B-positive Gaussian
block at seed 0 on both sides.

Bar, for the FP64 form and for the mixed FP32/FP64 form alike: eigenvalues
within 1e-9 relative of the oracle's FP64 solve, true residual <= tol on the
returned modes (recomputed with the oracle's operators), subspace angle
<= 1e-6 against the oracle's vectors for the modes set apart from the rest
of the spectrum (the first 7).
"""
import os
import sys

import numpy as np
import pytest

from oracle import bdg_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_fixtures as FX  # noqa: E402

pytestmark = pytest.mark.gpu

NEV, M, TOL = 8, 16, 1e-8


@pytest.fixture(scope="module")
def c1():
    fx = FX.load("c1_32")
    N = [int(v) for v in fx["N"]]
    L = [float(v) for v in fx["L"]]
    om = [float(v) for v in fx["omegas"]]
    g, gdd, rc, mu = float(fx["g"]), float(fx["gdd"]), float(fx["rc"]), float(fx["mu"])
    psi = fx["psi"]
    oc = O.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc)
    X0 = O.gaussian_block_bpositive(oc, M, 0)
    proj, _ = O.goldstone_projector(oc)
    ref = O.ilobpcg(oc, X0, NEV, 400, TOL, proj=proj, criterion=O.CONV_TRUE_RESIDUAL)
    assert ref.converged >= NEV
    return dict(N=N, L=L, om=om, g=g, gdd=gdd, rc=rc, mu=mu, psi=psi, oc=oc, X0=X0, ref=ref)


def _subspace_angle(A, Bm):
    qa, _ = np.linalg.qr(A.T)
    qb, _ = np.linalg.qr(Bm.T)
    s = np.linalg.svd(qa.conj().T @ qb, compute_uv=False)
    return float(np.arccos(np.clip(np.min(s), -1.0, 1.0)))


@pytest.mark.parametrize("precision", [0, 1])
def test_c1_gpu_matches_oracle(precision, c1, bdg):
    oc, ref = c1["oc"], c1["ref"]
    g = c1["g"]
    p = bdg.Problem(3, c1["N"], c1["L"])
    p.set_system()
    p.set_trap(O.harmonic_trap(oc, c1["om"]))
    p.set_wavefunction(c1["psi"])
    p.set_local_interactions(lambda n: g * n, lambda n: g * n)
    p.set_dipolar(c1["gdd"], [0.0, 0.0, 1.0], c1["rc"])
    p.set_mu(c1["mu"])
    p.set_solver_params(NEV, M, 400, TOL)
    p.set_initial_block(c1["X0"])
    p.set_goldstone_deflation(True)
    p.set_convergence(bdg.CONV_TRUE_RESIDUAL)
    p.set_precision(precision)
    assert p.solve() == 0
    assert p.converged() >= NEV
    ev = p.eigenvalues()[:NEV]
    rel = np.abs(ev - ref.eigvals[:NEV]) / np.abs(ref.eigvals[:NEV])
    assert np.all(rel < 1e-9), (ev, ref.eigvals[:NEV], rel)
    assert p.stats()["max_true_residual"] <= TOL
    X = p.block()[:NEV]
    tres = O.true_residual(oc, X, O.matmulLrep(oc, X), ev, NEV)
    assert np.all(tres <= 2 * TOL), tres
    # modes 8 and 9 lie 2e-4 apart (1.98089, 1.98127), so the span of the
    # first 8 is fixed only to residual / gap; the first 7 are 0.3 from the rest
    assert _subspace_angle(X[:7], ref.X[:7]) < 1e-6
    p.close()
