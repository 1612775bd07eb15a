"""GPU parity against the reference's own code (oracle/_ref).

* The reference's own C tests (tests/test_*.c of pstuermer/BDG_LOBPCG,
  unmodified), compiled against the product library libbdg_b200.so
  (oracle/_ref/tests_b200), pass on the GPU.  tests/test_bdg_3d_harmonic.c
  asserts that all nine excited modes of the isotropic oscillator lie at
  1.0 +- 5%; the analytic spectrum is 1 (x3) then 2 (x6), and the reference
  code itself fails that assertion (oracle build: modes 4-9 at 2.00000).
  Its output is checked against the analytic spectrum instead.
* The CUDA operators, given the fields the reference's own setup chain
  produced, match the reference's operators to 1e-12 relative (FP64) on the
  dipolar trap of the 32^3 benchmark config (stationary psi0), real and
  complex, and on the 64^3 grid of the mixed-precision config.
* The product's setup chain (trap, wavefunction, contact interactions,
  dipolar kernel and mean field on the GPU, mu) yields the reference's
  localTermK/M and preconditioner arrays to 1e-13.
* The initial blocks the GPU writes (PLANEWAVE, complex WF_WEIGHTED) match
  the reference's init switch to the rounding of sin, cos, log and sqrt
  (1e-14 relative), draw for draw.
* Solves: the GPU solve of the 32^3 benchmark config (nev 8, sizeSub 16,
  seed-0 block, true residual <= 1e-8, Goldstone chain deflated), FP64 and
  mixed FP32/FP64, against the reference's solve path on the same inputs:
  eigenvalues within 1e-9 relative, true residual <= tol, subspace angle of
  the first 7 modes <= 1e-6 (modes 8 and 9 lie 2e-4 apart).
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import bdg_oracle as O
from oracle import ref as R

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle build missing")]

HERE = os.path.dirname(os.path.abspath(__file__))
REL64 = 1e-12

C_TESTS = ["test_bdg_1d_uniform", "test_dipolar", "test_io", "test_kinetic", "test_matmulK", "test_matmulLrep",
           "test_matmulM", "test_matmulSwap", "test_precond", "test_setup"]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", autouse=True)
def _threads():
    R.set_threads(max(1, min(8, os.cpu_count() or 1)))


@pytest.mark.parametrize("name", C_TESTS)
def test_reference_c_test_on_product_library(name, bdg):
    exe = os.path.join(R.TESTS_B200_DIR, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert ", 0 failed" in r.stdout


def test_reference_harmonic_test_on_product_library(bdg):
    exe = os.path.join(R.TESTS_B200_DIR, "test_bdg_3d_harmonic")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    out = r.stdout
    assert "bdg_solve returned: 0" in out
    assert "converged: 10 / 10" in out
    ev = [float(v) for v in re.search(r"eigenvalues:((?: [-0-9.e+]+)+)", out).group(1).split()]
    assert abs(ev[0]) < 0.1  # the Goldstone mode
    assert all(abs(e - 1.0) < 0.05 for e in ev[1:4])
    assert all(abs(e - 2.0) < 0.05 for e in ev[4:10])
    # the only failing assertion is the one that expects 1.0 for modes 4-9
    fails = re.findall(r"\[FAIL\] line \d+: ([-0-9.e+]+) vs ([-0-9.e+]+)", out)
    assert len(fails) == 1 and abs(float(fails[0][0]) - 2.0) < 0.05 and float(fails[0][1]) == 1.0


def _fixture(name):
    p = os.path.join(HERE, "golden", f"{name}.npz")
    if not os.path.exists(p):
        pytest.skip(f"fixture {name} missing")
    f = np.load(p)
    return ([int(v) for v in f["N"]], [float(v) for v in f["L"]], [float(v) for v in f["omegas"]], float(f["g"]),
            float(f["gdd"]), float(f["rc"]), float(f["mu"]), f["psi"])


def _product_problem(bdg, N, L, om, g, gdd, rc, mu, psi, cplx=False):
    oc = O.Ctx(3, N, L, cplx)
    V = O.harmonic_trap(oc, om)
    p = bdg.Problem(3, N, L, complex_psi0=cplx)
    p.set_system()
    p.set_trap(V)
    p.set_wavefunction(psi)
    p.set_local_interactions(lambda n: g * n, lambda n: g * n)
    p.set_dipolar(gdd, [0.0, 0.0, 1.0], rc)
    p.set_mu(mu)
    return p


@pytest.mark.parametrize("case", ["c1_32-d", "c1_32-z", "c2_64-d"])
def test_operators_and_setup_match_reference(case, bdg):
    name, t = case.split("-")
    cplx = t == "z"
    N, L, om, g, gdd, rc, mu, psi = _fixture(name)
    if cplx:
        psi = psi * np.exp(0.7j)
    rp = R.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc, complex_psi0=cplx)
    # the product's setup chain against the reference's
    p = _product_problem(bdg, N, L, om, g, gdd, rc, mu, psi, cplx)
    K, M = p.local_terms()
    assert _rel(K, rp.field("localTermK")) < 1e-13
    assert _rel(M, rp.field("localTermM")) < 1e-13
    p.close()
    # the CUDA operators on the reference's fields
    gc = bdg.OperatorContext(3, N, L, cplx)
    for fld in ("localTermK", "localTermM", "precond_sqrtK", "precond_sqrtM"):
        gc.set(fld, rp.field(fld))
    gc.set("wf", psi)
    gc.set_scalar("mu", mu)
    gc.set_dipolar_kernel(gdd, [0.0, 0.0, 1.0], rc)
    gc.set_scalar("dipolar", 1)
    ops = R.RefOperators(rp)
    rng = np.random.default_rng(3)
    size = int(np.prod(N))
    for op in ops.OPS:
        n = (2 if op in ops.BLOCK else 1) * size
        x = rng.standard_normal(n)
        if cplx:
            x = x + 1j * rng.standard_normal(n)
        e = _rel(gc.apply(op, x), ops.apply(op, x))
        assert e < REL64, (op, e)
    rp.close()


def _init_pair(bdg, cplx, mode, hint, m=9):
    rng = np.random.default_rng(21)
    dim, N, L = 3, [16, 16, 32], [8.0, 6.0, 12.0]
    size = int(np.prod(N))
    psi = rng.random(size) + 0.1
    psi[::7] = 0.0
    if cplx:
        psi = psi * np.exp(1j * rng.random(size))
    rp = R.RefProblem(dim, N, L, cplx)
    rp.set_system()
    rp.set_wavefunction(psi)
    rp.set_mu(1.0)
    rp.set_solver_params(max(1, m // 2), m, 10, 1e-8)
    rp.L_.bdg_set_init_mode(rp.h, mode, None, C.c_void_p(hint) if hint else None)
    Xr = rp.initial_block()
    rp.close()
    p = bdg.Problem(dim, N, L, complex_psi0=cplx)
    p.set_system()
    p.set_wavefunction(psi)
    p.set_mu(1.0)
    p.set_solver_params(max(1, m // 2), m, 10, 1e-8)
    p.set_init_mode(mode, param=hint)
    return p, Xr


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("mode,hint", [(0, 0), (0, 1), (0, 2), (1, 0)])
def test_device_initial_block_matches_reference(bdg, cplx, mode, hint):
    if mode == 1 and not cplx:
        pytest.skip("the real WF_WEIGHTED block is time-seeded in the reference")
    torch = pytest.importorskip("torch")
    p, Xr = _init_pair(bdg, cplx, mode, hint)
    lib = bdg.lib()
    f = lib.bdg_fill_initial_block_device
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    assert p.device_context() is not None
    dev = torch.full((Xr.size * (2 if cplx else 1),), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert f(p._h, C.c_void_p(dev.data_ptr()), 0) == 0
    torch.cuda.synchronize()
    d = dev.cpu().numpy()
    if cplx:
        d = d.view(np.complex128)
    d = d.reshape(Xr.shape)
    assert np.all(np.isfinite(d))
    assert _rel(d, Xr) <= 1e-14
    p.close()


def _angles(A, Bm):
    """Largest principal angle between the row spaces of A and B."""
    qa, _ = np.linalg.qr(A.T)
    qb, _ = np.linalg.qr(Bm.T)
    s = np.linalg.svd(qa.conj().T @ qb, compute_uv=False)
    return float(np.arccos(np.clip(s.min(), -1.0, 1.0)))


@pytest.fixture(scope="module")
def c1_reference_solve():
    N, L, om, g, gdd, rc, mu, psi = _fixture("c1_32")
    nev, m, tol = 8, 16, 1e-8
    rp = R.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc)
    oc = O.Ctx(3, N, L)
    X0 = O.gaussian_block_bpositive(oc, m, 0)
    rp.set_solver_params(nev, m, 400, tol)
    rp.set_initial_block(X0)
    res = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    u, v = rp.modes()
    rp.close()
    assert res["converged"] >= nev
    return dict(N=N, L=L, om=om, g=g, gdd=gdd, rc=rc, mu=mu, psi=psi, nev=nev, m=m, tol=tol, X0=X0,
                eig=res["eigvals"], iters=res["iterations"], v=v)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_c1_solve_matches_reference_solve(bdg, c1_reference_solve, precision):
    r = c1_reference_solve
    p = _product_problem(bdg, r["N"], r["L"], r["om"], r["g"], r["gdd"], r["rc"], r["mu"], r["psi"])
    p.set_solver_params(r["nev"], r["m"], 400, r["tol"])
    p.set_initial_block(r["X0"])
    p.set_goldstone_deflation(True)
    p.set_convergence(bdg.CONV_TRUE_RESIDUAL)
    p.set_precision(bdg.PREC_MIXED if precision == "mixed" else bdg.PREC_F64)
    assert p.solve() == 0
    nev = r["nev"]
    assert p.converged() >= nev
    ev = p.eigenvalues()[:nev]
    rel = np.abs(ev - r["eig"]) / np.abs(r["eig"])
    assert np.all(rel < 1e-9), (ev, r["eig"])
    st = p.stats()
    assert st["max_true_residual"] <= r["tol"]
    v = p.modes_v()
    assert _angles(v[:7], r["v"][:7]) <= 1e-6
    p.close()


def test_c1_complex_solve_matches_reference_solve(bdg):
    """The complex (_z) path: psi0 = e^{0.7 i} x the stationary 32^3 state (a
    genuinely complex condensate with the real problem's spectrum), complex
    N(0,1) block with v = u at seed 2, true residual <= 1e-8, Goldstone chain
    deflated; GPU against the reference's complex solve path (z_ilobpcg of
    the oracle build): eigenvalues 1e-9, true residual <= tol, and the same
    eigenvalues as the real problem."""
    N, L, om, g, gdd, rc, mu, psi = _fixture("c1_32")
    psi_z = psi * np.exp(0.7j)
    nev, m, tol = 8, 16, 1e-8
    oc = O.Ctx(3, N, L, True)
    X0 = O.gaussian_block_bpositive(oc, m, 2)
    rp = R.build_problem(N, L, om, g, gdd, psi_z, mu, Rc=rc, complex_psi0=True)
    rp.set_solver_params(nev, m, 400, tol)
    rp.set_initial_block(X0)
    ref = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    rp.close()
    assert ref["converged"] >= nev
    p = _product_problem(bdg, N, L, om, g, gdd, rc, mu, psi_z, cplx=True)
    p.set_solver_params(nev, m, 400, tol)
    p.set_initial_block(X0)
    p.set_goldstone_deflation(True)
    p.set_convergence(bdg.CONV_TRUE_RESIDUAL)
    assert p.solve() == 0 and p.converged() >= nev
    ev = p.eigenvalues()[:nev]
    assert np.all(np.abs(ev - ref["eigvals"]) / np.abs(ref["eigvals"]) < 1e-9), (ev, ref["eigvals"])
    assert p.stats()["max_true_residual"] <= tol
    real = np.load(os.path.join(HERE, "golden", "c1_32_solve.npz"))["eigvals"][:nev]
    assert np.all(np.abs(ev - real) / real < 1e-9)
    p.close()
