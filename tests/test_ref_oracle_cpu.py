"""The oracle pinned on the reference's own code (CPU).

``oracle/_ref`` is pstuermer/BDG_LOBPCG's own src/*.c compiled unmodified by
``oracle/Makefile`` against the project's stand-ins for its absent
dependencies (FFTW3-subset CPU FFT, the external iLOBPCG restated in C,
OpenBLAS).  These tests check:

* the reference's own unit and solver tests (tests/test_*.c, unmodified) pass
  on that build -- all but tests/test_bdg_3d_harmonic.c, whose assertion that
  all nine excited oscillator modes lie at 1.0 +- 5% fails on the reference
  code itself (modes 4-9 are the analytic 2.0; 3.5 min on 8 cores, so it is
  run by the GPU suite against the product library instead);
* the numpy oracle's setup fields and all nine operators agree with the
  reference's to 1e-13 relative (FP64) on the dipolar trap of the 32^3
  benchmark config with its stationary psi0 (real path) and on a complex psi0;
* the init-mode restatement is bit-exact against the block the reference's
  init switch writes (PLANEWAVE, real path, every geometry hint) and within
  rounding of cabs on the complex path (PLANEWAVE and WF_WEIGHTED);
* the product library's own host fill of those blocks is bit-identical to
  the reference's;
* the numpy oracle's iLOBPCG and the reference's solve path (bdg_solve ->
  solver.c -> restated iLOBPCG on the reference operators) reach the same
  eigenvalues (1e-12) on the 16^3 dipolar problem.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import bdg_oracle as O
from oracle import ref as R

HERE = os.path.dirname(os.path.abspath(__file__))

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle build missing (make -C oracle)")

FAST_C_TESTS = ["test_bdg_1d_uniform", "test_dipolar", "test_io", "test_kinetic", "test_matmulK",
                "test_matmulLrep", "test_matmulM", "test_matmulSwap", "test_precond", "test_setup"]


@pytest.fixture(scope="module", autouse=True)
def _threads():
    R.set_threads(1)


@pytest.mark.parametrize("name", FAST_C_TESTS)
def test_reference_c_test_passes_on_oracle_build(name):
    exe = os.path.join(R.TESTS_DIR, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert ", 0 failed" in r.stdout


def _c1():
    f = np.load(os.path.join(HERE, "golden", "c1_32.npz"))
    N = [int(v) for v in f["N"]]
    L = [float(v) for v in f["L"]]
    om = [float(v) for v in f["omegas"]]
    return N, L, om, float(f["g"]), float(f["gdd"]), float(f["rc"]), float(f["mu"]), f["psi"]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("cplx", [False, True])
def test_operators_match_reference_build(cplx):
    N, L, om, g, gdd, rc, mu, psi = _c1()
    if cplx:
        psi = psi * np.exp(0.7j)
    oc = O.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc, complex_psi0=cplx)
    rp = R.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc, complex_psi0=cplx)
    for fld in ("localTermK", "localTermM", "precond_sqrtK", "precond_sqrtM", "longRngInt", "k2"):
        assert _rel(rp.field(fld), getattr(oc, fld).reshape(-1)) < 1e-13, fld
    ops = R.RefOperators(rp)
    rng = np.random.default_rng(1)
    for op in ops.OPS:
        n = (2 if op in ops.BLOCK else 1) * oc.size
        x = rng.standard_normal((2, n))
        if cplx:
            x = x + 1j * rng.standard_normal((2, n))
        assert _rel(ops.apply(op, x), getattr(O, op)(oc, x)) < 1e-13, op
    rp.close()


def _init_problem(dim, N, L, cplx, m, seed):
    rng = np.random.default_rng(seed)
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
    oc = O.Ctx(dim, N, L, cplx)
    O.set_system(oc)
    O.set_wavefunction(oc, psi)
    return rp, oc, psi


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("hint", [0, 1, 2])
@pytest.mark.parametrize("shape", ["3d", "1d_noise"])
def test_planewave_block_matches_reference(cplx, hint, shape):
    dim, N, L, m = (3, [16, 16, 32], [8.0, 6.0, 12.0], 9) if shape == "3d" else (1, [8], [4.0], 30)
    rp, oc, _ = _init_problem(dim, N, L, cplx, m, 5)
    rp.L_.bdg_set_init_mode(rp.h, R.BDG_INIT_PLANEWAVE, None, C.c_void_p(hint) if hint else None)
    Xr = rp.initial_block()
    Xo = O.planewave_block(oc, m, hint)
    if cplx:
        assert _rel(Xo, Xr) < 1e-15
    else:
        assert np.array_equal(Xo, Xr)
    rp.close()


def test_wf_weighted_complex_block_matches_reference():
    rp, oc, _ = _init_problem(3, [8, 8, 8], [5.0] * 3, True, 6, 7)
    rp.set_init_mode(R.BDG_INIT_WF_WEIGHTED)
    Xr = rp.initial_block()
    assert _rel(O.wf_weighted_block_z(oc, 6), Xr) < 1e-15
    rp.close()


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("mode,hint", [(0, 0), (0, 1), (0, 2), (1, 0)])
def test_library_host_fill_is_bit_identical_to_reference(bdg, cplx, mode, hint):
    if mode == 1 and not cplx:
        pytest.skip("the real WF_WEIGHTED block is time-seeded in the reference")
    dim, N, L, m = 3, [16, 16, 32], [8.0, 6.0, 12.0], 9
    rp, _, psi = _init_problem(dim, N, L, cplx, m, 11)
    rp.L_.bdg_set_init_mode(rp.h, mode, None, C.c_void_p(hint) if hint else None)
    Xr = rp.initial_block()
    p = bdg.Problem(dim, N, L, complex_psi0=cplx)
    p.set_system()
    p.set_wavefunction(psi)
    p.set_mu(1.0)
    p.set_solver_params(max(1, m // 2), m, 10, 1e-8)
    p.set_init_mode(mode, param=hint)
    lib = bdg.lib()
    lib.bdg_fill_initial_block.restype = None
    lib.bdg_fill_initial_block.argtypes = [C.c_void_p, C.c_void_p]
    host = np.zeros(Xr.size, dtype=Xr.dtype)
    lib.bdg_fill_initial_block(p._h, host.ctypes.data)
    assert np.array_equal(host.reshape(Xr.shape), Xr)
    p.close()
    rp.close()


def test_oracle_solve_matches_reference_solve_path():
    f = np.load(os.path.join(HERE, "golden", "gs16.npz"))
    N = [int(v) for v in f["N"]]
    L = [float(v) for v in f["L"]]
    om = [float(v) for v in f["omegas"]]
    g, gdd, rc, mu, psi = float(f["g"]), float(f["gdd"]), float(f["rc"]), float(f["mu"]), f["psi"]
    nev, m, tol = 4, 8, 1e-8
    oc = O.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc)
    X0 = O.gaussian_block_bpositive(oc, m, 0)
    proj, _ = O.goldstone_projector(oc)
    ro = O.ilobpcg(oc, X0, nev, 400, tol, proj=proj, criterion=O.CONV_TRUE_RESIDUAL)
    rp = R.build_problem(N, L, om, g, gdd, psi, mu, Rc=rc)
    rp.set_solver_params(nev, m, 400, tol)
    rp.set_initial_block(X0)
    res = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    assert res["converged"] >= nev and ro.converged >= nev
    rel = np.abs(res["eigvals"] - ro.eigvals[:nev]) / np.abs(ro.eigvals[:nev])
    assert np.all(rel < 1e-12), (res["eigvals"], ro.eigvals[:nev])
    assert abs(res["iterations"] - ro.iters) <= 3
    # the reference's modes are the converged Ritz vectors: true residual <= tol
    u, v = rp.modes()
    for j in range(nev):
        Mv = O.matmulM(oc, v[j])
        r = O.matmulK(oc, Mv) - res["eigvals"][j] ** 2 * v[j]
        assert np.linalg.norm(r) / np.linalg.norm(v[j]) <= tol
    rp.close()


def test_reference_solve_path_p_normalisation_option():
    """The oracle build's iLOBPCG with the projected P SVQB-normalised
    (normalize_p) and without (the default, as on the GPU): same eigenvalues
    (1e-12) and iteration counts within one on the 16^3 dipolar problem."""
    f = np.load(os.path.join(HERE, "golden", "gs16.npz"))
    N = [int(v) for v in f["N"]]
    L = [float(v) for v in f["L"]]
    om = [float(v) for v in f["omegas"]]
    oc = O.Ctx(3, N, L)
    X0 = O.gaussian_block_bpositive(oc, 8, 0)
    out = []
    for norm in (False, True):
        rp = R.build_problem(N, L, om, float(f["g"]), float(f["gdd"]), f["psi"], float(f["mu"]), Rc=float(f["rc"]))
        rp.set_solver_params(4, 8, 400, 1e-8)
        rp.set_initial_block(X0)
        out.append(rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True, normalize_p=norm))
        rp.close()
    assert all(r["converged"] >= 4 for r in out)
    assert np.all(np.abs(out[0]["eigvals"] - out[1]["eigvals"]) / np.abs(out[1]["eigvals"]) < 1e-12)
    assert abs(int(out[0]["iterations"]) - int(out[1]["iterations"])) <= 1
