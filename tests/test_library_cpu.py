"""Host-side checks of the C library that need no GPU: the shared library
loads, exports every entry point declared in include/*.h, and the host setup
logic (trap, wavefunction, interactions, mu, reset, state errors, I/O
formats) behaves as the reference's tests/test_setup.c and tests/test_io.c
require."""
import math
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for fn in ("bdg/bdg.h", "bdg/bdg_b200.h", "bdg/bdg_cuda.h", "bdg/bdg_internal.h"):
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"static inline[^{]*\{.*?\n\}", "", src, flags=re.S)
        src = re.sub(r"^\s*#.*$", "", src, flags=re.M)  # macros (the FFTW-name compatibility)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{]*)\)\s*;", src):
            name = m.group(1)
            if name in ("if", "while", "for", "sizeof", "return", "void", "int", "double") or name.startswith("BDG_"):
                continue
            names.add(name)
    return sorted(names)


def test_library_exports_declared_symbols(bdg):
    L = bdg.lib()
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # the 22 public functions of the reference API (include/bdg/bdg.h)
    public = ["bdg_alloc", "bdg_free", "bdg_reset", "bdg_set_system", "bdg_set_trap", "bdg_set_wavefunction",
              "bdg_set_local_interactions", "bdg_set_mu", "bdg_set_dipolar", "bdg_set_solver_params",
              "bdg_set_init_mode", "bdg_reuse_modes", "bdg_solve", "bdg_converged", "bdg_eigenvalues",
              "bdg_modes_u", "bdg_modes_v", "bdg_load_wavefunction", "bdg_load_wavefunction_fmt",
              "bdg_write_eigenvalues", "bdg_write_mode_u", "bdg_write_mode_v"]
    assert all(hasattr(L, n) for n in public)
    assert len(public) == 22


def test_no_cpu_fallback_without_gpu(bdg):
    """The operators need the GPU; without one they fail loudly (the
    library exits with its error) instead of computing on the host."""
    if bdg.gpu_available():
        pytest.skip("a GPU is present")
    code = ("import numpy as np, bdg_lobpcg_b200 as B\n"
            "c = B.OperatorContext(1, [16], [1.0])\n"
            "c.apply('kinetic', np.ones(16))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "GPU apply failed" in r.stderr


def _harm(omega):
    return lambda dim, r: 0.5 * omega * omega * sum(x * x for x in r[:dim])


def test_k_tables(bdg):
    """tests/test_setup.c:49-190: k_size and kx2 for r2c and c2c."""
    c = bdg.OperatorContext(3, [8, 6, 4], [1.0, 2.0, 3.0], False)
    assert c.k_size == 5 * 6 * 4
    dk = 2 * math.pi / 2.0
    kx2 = c.kx2(1)
    assert np.allclose(kx2, (dk * np.array([0, 1, 2, 3, -2, -1])) ** 2, atol=1e-12)
    cz = bdg.OperatorContext(2, [16, 8], [1.0, 1.0], True)
    assert cz.k_size == 128


def test_trap_grid_and_callback(bdg):
    """tests/test_setup.c:299-360: V at r_i = (i - N/2) L / N, added to both
    local terms; repeated calls add (trap_additive)."""
    p = bdg.Problem(2, [8, 6], [4.0, 3.0])
    p.set_system()
    p.set_trap(_harm(2.0))
    K, M = p.local_terms()
    x = (np.arange(8) - 4.0) * 0.5
    y = (np.arange(6) - 3.0) * 0.5
    Y, X = np.meshgrid(y, x, indexing="ij")
    exp = (0.5 * 4.0 * (X * X + Y * Y)).reshape(-1)
    assert np.allclose(K, exp, atol=1e-10) and np.allclose(M, exp, atol=1e-10)
    p.set_trap(exp)
    K2, _ = p.local_terms()
    assert np.allclose(K2, 2 * exp, atol=1e-10)
    assert p.state() & bdg.HAS_TRAP


def test_interactions_and_mu(bdg):
    """tests/test_setup.c:404-530: contact K += g n, M += 3 g n; set_mu
    builds 1/sqrt(max(1e-8, lt)) before subtracting mu."""
    p = bdg.Problem(1, [8], [4.0])
    p.set_system()
    p.set_trap(_harm(1.0))
    p.set_wavefunction(np.ones(8))
    p.set_local_interactions_callback(lambda n: 1.0 * n, lambda n: 1.0 * n)
    K0, M0 = p.local_terms()
    p.set_mu(3.0)
    K, M = p.local_terms()
    assert np.allclose(K, K0 - 3.0, atol=1e-14) and np.allclose(M, M0 - 3.0, atol=1e-14)
    c = p.ctx
    pK = np.ctypeslib.as_array(c.precond_sqrtK, shape=(8,))
    assert np.allclose(pK, 1.0 / np.sqrt(np.fmax(1e-8, K0)), atol=1e-14)
    assert c.mu == 3.0
    x = (np.arange(8) - 4.0) * 0.5
    assert np.allclose(M0, 0.5 * x * x + 3.0, atol=1e-14)


def test_wavefunction_copy(bdg):
    """tests/test_setup.c:365-400: real and complex copies."""
    p = bdg.Problem(1, [8], [1.0])
    p.set_system()
    w = np.sin(2 * math.pi * np.arange(8) / 8)
    p.set_wavefunction(w)
    assert np.allclose(p.wavefunction(), w) and p.state() & bdg.HAS_WF
    pz = bdg.Problem(1, [8], [1.0], True)
    pz.set_system()
    wz = np.arange(8) + 1j * (8 - np.arange(8))
    pz.set_wavefunction(wz)
    assert np.allclose(pz.wavefunction(), wz)


def test_reset_keeps_system(bdg):
    """tests/test_setup.c:602-699: reset clears physics, keeps the grid."""
    p = bdg.Problem(1, [8], [4.0])
    p.set_system()
    p.set_trap(_harm(1.0))
    p.set_wavefunction(np.ones(8))
    p.set_local_interactions(lambda n: n, lambda n: n)
    p.set_mu(2.0)
    p.raw.state
    L = bdg.lib()
    L.bdg_reset(p._h)
    assert p.state() == bdg.HAS_SYSTEM
    K, M = p.local_terms()
    assert np.all(K == 0) and np.all(M == 0)
    assert not p.ctx.wf and not p.ctx.precond_sqrtK
    assert p.ctx.mu == 0.0 and p.ctx.k2
    p.set_trap(_harm(3.0))
    p.set_wavefunction(np.full(8, 0.5))
    p.set_local_interactions(lambda n: 5.0 * n, lambda n: 5.0 * n)
    p.set_mu(1.0)
    K, M = p.local_terms()
    x = (np.arange(8) - 4.0) * 0.5
    V = 0.5 * 9.0 * x * x
    assert np.allclose(K, V + 5 * 0.25 - 1, atol=1e-12)
    assert np.allclose(M, V + 15 * 0.25 - 1, atol=1e-12)


DEATH = {
    "trap_without_system": "p = B.Problem(1,[8],[1.0]); p.set_trap(np.zeros(8))",
    "wf_without_system": "p = B.Problem(1,[8],[1.0]); p.set_wavefunction(np.zeros(8))",
    "interactions_without_wf": "p = B.Problem(1,[4],[1.0]); p.set_system(); "
                               "B.lib().bdg_set_local_interactions_grid(p._h, B._dptr(np.zeros(4)), B._dptr(np.zeros(4)))",
    "interactions_twice": "p = B.Problem(1,[4],[1.0]); p.set_system(); p.set_wavefunction(np.ones(4)); "
                          "p.set_local_interactions(lambda n: n, lambda n: n); p.set_local_interactions(lambda n: n, lambda n: n)",
    "dipolar_not_3d": "p = B.Problem(1,[4],[1.0]); p.set_system(); p.set_wavefunction(np.ones(4)); p.set_dipolar(1.0,[0,0,1],1.0)",
    "dipolar_after_mu": "p = B.Problem(3,[4,4,4],[1.0]*3); p.set_system(); p.set_wavefunction(np.ones(64)); p.set_mu(1.0); p.set_dipolar(1.0,[0,0,1],1.0)",
    "wf_wrong_size": "p = B.Problem(1,[8],[1.0]); p.set_system(); B.lib().bdg_set_wavefunction(p._h, B._ptr(np.ones(8)), 7)",
    "solve_without_mu": "p = B.Problem(1,[8],[1.0]); p.set_system(); p.solve()",
}


@pytest.mark.parametrize("name", sorted(DEATH))
def test_state_errors_exit_failure(name, bdg):
    """tests/test_setup.c:532-600: misuse exits with EXIT_FAILURE (run in a
    child process, as the reference does with fork)."""
    code = "import numpy as np, bdg_lobpcg_b200 as B\n" + DEATH[name] + "\n"
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 1, (r.returncode, r.stderr[-400:])
    assert "ERROR" in r.stderr


def test_io_roundtrip_and_codes(bdg, tmp_path):
    """tests/test_io.c:45-200: load "re im" lines; missing file -1; short
    file -2; write_* without results -3."""
    f = tmp_path / "wf.dat"
    f.write_text("1.0 0.0\n2.0 0.0\n3.0 0.0\n4.0 0.0\n")
    p = bdg.Problem(1, [4], [1.0])
    p.set_system()
    assert p.load_wavefunction(str(f)) == 0
    assert np.allclose(p.wavefunction(), [1, 2, 3, 4])
    assert p.load_wavefunction(str(tmp_path / "missing.dat")) == -1
    g = tmp_path / "short.dat"
    g.write_text("1.0 0.0\n")
    q = bdg.Problem(1, [4], [1.0])
    q.set_system()
    assert q.load_wavefunction(str(g)) == -2
    fz = tmp_path / "wfz.dat"
    fz.write_text("1.0 0.5\n2.0 -0.5\n")
    pz = bdg.Problem(1, [2], [1.0], True)
    pz.set_system()
    assert pz.load_wavefunction(str(fz)) == 0
    assert np.allclose(pz.wavefunction(), [1 + 0.5j, 2 - 0.5j])
    assert p.write_eigenvalues(str(tmp_path / "ev.dat")) == -3
    assert p.write_mode_u(0, str(tmp_path / "m")) == -3
    assert p.reuse_modes(0.1) == -3


def test_init_block_planewave_host(bdg):
    """src/solver.c:214-259: the planewave initial block (u = v, cos/sin of
    the lowest |k| times |psi0|) is filled on the host before upload."""
    L = bdg.lib()
    import ctypes as C

    p = bdg.Problem(1, [16], [2 * math.pi])
    p.set_system()
    p.set_wavefunction(np.ones(16))
    L.bdg_set_solver_params(p._h, 2, 4, 10, 1e-6)
    fill = L.bdg_fill_initial_block
    fill.argtypes = [C.c_void_p, C.c_void_p]
    S = np.zeros((4, 32))
    fill(p._h, S.ctypes.data_as(C.c_void_p))
    x = np.arange(16) * 2 * math.pi / 16
    assert np.allclose(S[:, :16], S[:, 16:])
    assert np.allclose(S[0, :16], 1.0, atol=1e-4)  # k = 0 cos
    assert np.allclose(np.abs(S[1, :16]), np.abs(np.sin(x)), atol=1e-4)


def test_public_headers_compile_as_c11_and_cpp(tmp_path):
    """The C ABI headers compile as the reference compiles its sources
    (-std=c11, Makefile:3) with -Wall -Wextra -pedantic -Werror, and as C++17."""
    import shutil
    import subprocess

    if not shutil.which("gcc") or not shutil.which("g++"):
        pytest.skip("no host compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "hdr.c"
    src.write_text("\n".join(f'#include "bdg/{h}"' for h in
                             ("bdg.h", "bdg_b200.h", "bdg_cuda.h", "bdg_learn.h", "bdg_internal.h", "memory.h"))
                   + "\nint main(void) { return 0; }\n")
    for cmd in (["gcc", "-std=c11", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-I", inc, str(src)],
                ["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-x", "c++", "-I", inc, str(src)]):
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_set_initial_block_borrowed(bdg, capfd):
    """bdg_set_initial_block: the host fill copies the caller's block exactly
    (real and complex); a shape that is not the problem's is refused (-2, a
    ValueError in the binding); a sizeSub changed afterwards yields a zero
    block and a message instead of reading past the caller's array."""
    import ctypes as C

    lib = bdg.lib()
    lib.bdg_fill_initial_block.restype = None
    lib.bdg_fill_initial_block.argtypes = [C.c_void_p, C.c_void_p]
    for cplx in (False, True):
        p = bdg.Problem(1, [8], [4.0], cplx)
        p.set_system()
        p.set_solver_params(2, 4, 10, 1e-6)
        rng = np.random.default_rng(4)
        X = rng.standard_normal((4, 16)) + (1j * rng.standard_normal((4, 16)) if cplx else 0)
        p.set_initial_block(X)
        out = np.zeros(X.size * (2 if cplx else 1))
        lib.bdg_fill_initial_block(p._h, out.ctypes.data)
        got = out.view(np.complex128) if cplx else out
        assert np.array_equal(got.reshape(4, 16), X)
        with pytest.raises(ValueError):
            p.set_initial_block(X[:3])
        p.set_solver_params(2, 5, 10, 1e-6)  # sizeSub no longer matches the borrowed block
        out2 = np.full(16 * 5 * (2 if cplx else 1), 7.0)
        lib.bdg_fill_initial_block(p._h, out2.ctypes.data)
        assert np.all(out2 == 0.0)
        assert "bdg_set_initial_block" in capfd.readouterr().err
        p.close()
