"""ctypes binding of the oracle build of the reference library.

TEST INFRASTRUCTURE ONLY.  ``oracle/_ref/libbdg_ref.so`` is pstuermer/
BDG_LOBPCG's own ``src/*.c``, compiled unmodified by ``oracle/Makefile``
against the project's stand-ins for its absent dependencies (an FFTW3-subset
CPU FFT, the external LOBPCG library's linop/iLOBPCG restated in C, OpenBLAS
from scipy).  Only ``tests/``, ``__graft_entry__`` and bench.py's CPU
baseline / reference legs use this module, as the checker and as the timed
reference CPU path.

* ``RefProblem`` drives the reference's public API (include/bdg/bdg.h):
  bdg_alloc -> set_system -> set_trap -> set_wavefunction ->
  set_local_interactions -> set_dipolar -> set_mu -> set_solver_params ->
  set_init_mode -> bdg_solve, the chain of the reference's examples
  (examples/3d_jens.c:53-67).  Trap and contact interactions go through C
  callbacks (a table lookup and U(n) = g n); a prepared initial block goes
  through BDG_INIT_CUSTOM.
* ``RefOperators`` calls the reference's single-column operators
  (src/bdg_internal.h:159-215) on the context of a RefProblem, the way the
  reference's unit tests do.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libbdg_ref.so")
TESTS_DIR = os.path.join(HERE, "_ref", "tests")
TESTS_B200_DIR = os.path.join(HERE, "_ref", "tests_b200")

BDG_INIT_PLANEWAVE, BDG_INIT_WF_WEIGHTED, BDG_INIT_REUSE, BDG_INIT_CUSTOM = 0, 1, 2, 3
CONV_BACKWARD, CONV_TRUE_RESIDUAL = 0, 1

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    """Load libbdg_ref.so once (RTLD_LOCAL: its symbols, the same names as
    the product library's, stay private to it)."""
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise RuntimeError(f"oracle build missing: {LIB_PATH} (make -C oracle)")
    L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
    vp, u64, f64, i32 = C.c_void_p, C.c_uint64, C.c_double, C.c_int
    sig = {
        "bdg_alloc": (vp, [u64, C.POINTER(u64), C.POINTER(f64), i32]),
        "bdg_free": (None, [C.POINTER(vp)]),
        "bdg_set_system": (None, [vp]),
        "bdg_set_trap": (None, [vp, vp, vp]),
        "bdg_set_wavefunction": (None, [vp, vp, u64]),
        "bdg_set_local_interactions": (None, [vp, vp, vp, vp]),
        "bdg_set_mu": (None, [vp, f64]),
        "bdg_set_dipolar": (None, [vp, f64, C.POINTER(f64), f64]),
        "bdg_set_solver_params": (None, [vp, u64, u64, u64, f64]),
        "bdg_set_init_mode": (None, [vp, i32, vp, vp]),
        "bdg_solve": (i32, [vp]),
        "bdg_converged": (u64, [vp]),
        "bdg_eigenvalues": (vp, [vp]),
        "bdg_modes_u": (vp, [vp]),
        "bdg_modes_v": (vp, [vp]),
        "ref_helper_ctx": (vp, [vp]),
        "ref_helper_field": (vp, [vp, C.c_char_p]),
        "ref_helper_get": (f64, [vp, C.c_char_p]),
        "ref_helper_set": (None, [vp, C.c_char_p, f64]),
        "ref_helper_anorm": (f64, [vp]),
        "ilobpcg_shim_set": (None, [i32, i32, i32, f64, f64, i32, f64]),
        "ilobpcg_shim_threads": (None, [i32]),
        "ilobpcg_shim_set_pnorm": (None, [i32]),
        "ilobpcg_shim_timeline": (i32, [C.POINTER(f64), i32, C.POINTER(i32), C.POINTER(i32)]),
        "ilobpcg_shim_history": (i32, [i32, i32, C.POINTER(f64), C.POINTER(f64)]),
        "ilobpcg_shim_capture_init": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    for op in ("kinetic", "matmulK", "matmulM", "matmulLrep", "matmulSwap", "precondK", "precondM",
               "precondLrep", "dipolar_conv"):
        for t in ("d", "z"):
            fn = getattr(L, f"{op}_{t}")
            fn.restype = None
            fn.argtypes = [vp, vp, vp]
    _lib = L
    return L


def set_threads(n):
    lib().ilobpcg_shim_threads(int(n))


class _TrapTable(C.Structure):
    _fields_ = [("V", C.c_void_p), ("next", C.c_uint64)]


class RefProblem:
    """A bdg_t of the oracle build, set up through the reference's API."""

    def __init__(self, dim, N, L, complex_psi0=False):
        self.L_ = lib()
        self.dim = dim
        self.N = [int(v) for v in N]
        self.Lb = [float(v) for v in L]
        self.cplx = bool(complex_psi0)
        self.size = int(np.prod(self.N))
        Na = (C.c_uint64 * dim)(*self.N)
        La = (C.c_double * dim)(*self.Lb)
        self.h = C.c_void_p(self.L_.bdg_alloc(dim, Na, La, 1 if complex_psi0 else 0))
        self._keep = []

    def close(self):
        if self.h:
            self.L_.bdg_free(C.byref(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ctx(self):
        return C.c_void_p(self.L_.ref_helper_ctx(self.h))

    def set_system(self):
        self.L_.bdg_set_system(self.h)

    def set_trap(self, V):
        V = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(-1))
        t = _TrapTable(V.ctypes.data, 0)
        fn = C.cast(self.L_.ref_cb_trap_table, C.c_void_p)
        self.L_.bdg_set_trap(self.h, fn, C.byref(t))
        assert t.next == self.size

    def set_wavefunction(self, psi):
        psi = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128 if self.cplx else np.float64).reshape(-1))
        self.L_.bdg_set_wavefunction(self.h, psi.ctypes.data, self.size)

    def set_contact(self, g):
        gv = C.c_double(float(g))
        self._keep.append(gv)
        fn = C.cast(self.L_.ref_cb_contact, C.c_void_p)
        self.L_.bdg_set_local_interactions(self.h, fn, fn, C.byref(gv))

    def set_dipolar(self, g_ddi, direction, Rc):
        d = (C.c_double * 3)(*[float(v) for v in direction])
        self.L_.bdg_set_dipolar(self.h, float(g_ddi), d, float(Rc))

    def set_mu(self, mu):
        self.L_.bdg_set_mu(self.h, float(mu))

    def set_solver_params(self, nev, sizeSub, maxIter, tol):
        self.L_.bdg_set_solver_params(self.h, int(nev), int(sizeSub), int(maxIter), float(tol))
        self.nev, self.m = int(nev), int(sizeSub)

    def set_init_mode(self, mode):
        self.L_.bdg_set_init_mode(self.h, int(mode), None, None)

    def set_initial_block(self, X):
        """X: (m, n) rows = columns of the n x m column-major block."""
        dt = np.complex128 if self.cplx else np.float64
        X = np.ascontiguousarray(np.asarray(X, dtype=dt))
        self._x0 = X
        fn = C.cast(self.L_.ref_cb_init_copy, C.c_void_p)
        self.L_.bdg_set_init_mode(self.h, BDG_INIT_CUSTOM, fn, C.c_void_p(X.ctypes.data))

    def initial_block(self):
        """The block the reference's init switch writes (src/solver.c:167-259,
        :321-414) for the current init mode, as (m, n) rows."""
        n = 2 * self.size
        dt = np.complex128 if self.cplx else np.float64
        out = np.zeros((self.m, n), dtype=dt)
        self.L_.ilobpcg_shim_capture_init(C.c_void_p(out.ctypes.data))
        self.L_.bdg_solve(self.h)
        return out

    def solve(self, criterion=CONV_BACKWARD, deflate=False, lock=True, guard=1e-4, guard_strict=1e-12,
              stall_win=10, true_gate=1e-7, normalize_p=False):
        self.L_.ilobpcg_shim_set(int(criterion), 1 if deflate else 0, 1 if lock else 0, guard, guard_strict,
                                 stall_win, true_gate)
        self.L_.ilobpcg_shim_set_pnorm(1 if normalize_p else 0)
        rc = self.L_.bdg_solve(self.h)
        if rc != 0:
            raise RuntimeError(f"bdg_solve (oracle build) returned {rc}")
        return self.result()

    def result(self):
        cap = 8192
        t = (C.c_double * cap)()
        it, nc = C.c_int(), C.c_int()
        nt = self.L_.ilobpcg_shim_timeline(t, cap, C.byref(it), C.byref(nc))
        ev = np.ctypeslib.as_array(C.cast(self.L_.bdg_eigenvalues(self.h), C.POINTER(C.c_double)),
                                   shape=(self.nev,)).copy()
        return {"eigvals": ev, "converged": int(self.L_.bdg_converged(self.h)), "iterations": it.value,
                "timeline": np.array(t[: min(nt, cap)])}

    def history(self, it):
        lam = (C.c_double * self.nev)()
        res = (C.c_double * self.nev)()
        n = self.L_.ilobpcg_shim_history(int(it), self.nev, lam, res)
        return np.array(lam[:]), np.array(res[:]), n

    def modes(self):
        dt = np.complex128 if self.cplx else np.float64
        ct = C.c_double if not self.cplx else C.c_double * 2
        out = []
        for fn in (self.L_.bdg_modes_u, self.L_.bdg_modes_v):
            p = fn(self.h)
            a = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)),
                                      shape=(self.nev * self.size * (2 if self.cplx else 1),))
            out.append(a.view(dt).reshape(self.nev, self.size).copy())
        return out

    def field(self, name, count=None, dtype=np.float64):
        p = self.L_.ref_helper_field(self.ctx, name.encode())
        if not p:
            return None
        if count is None:
            count = self.size if name not in ("k2", "longRngInt") else int(self.L_.ref_helper_get(self.ctx, b"k_size"))
        nd = 2 if dtype == np.complex128 else 1
        a = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(count * nd,))
        return a.view(dtype).copy()

    def anorm(self):
        return float(self.L_.ref_helper_anorm(self.ctx))


class RefOperators:
    """The reference's single-column operators on the context of a RefProblem."""

    OPS = ("kinetic", "matmulK", "matmulM", "matmulLrep", "matmulSwap", "precondK", "precondM", "precondLrep",
           "dipolar_conv")
    BLOCK = {"matmulLrep", "matmulSwap", "precondLrep"}

    def __init__(self, problem: RefProblem):
        self.p = problem

    def apply(self, op, x):
        """x: one column or (ncol, len) rows; len = size, or 2*size for the
        block operators."""
        p = self.p
        fn = getattr(p.L_, f"{op}_{'z' if p.cplx else 'd'}")
        dt = np.complex128 if p.cplx else np.float64
        x = np.asarray(x, dtype=dt)
        single = x.ndim == 1
        X = np.ascontiguousarray(x.reshape(1, -1) if single else x)
        n = (2 if op in self.BLOCK else 1) * p.size
        if X.shape[1] != n:
            raise ValueError(f"{op}: column length {X.shape[1]} != {n}")
        Y = np.zeros_like(X)
        ctx = p.ctx
        for j in range(X.shape[0]):
            fn(ctx, C.c_void_p(X[j].ctypes.data), C.c_void_p(Y[j].ctypes.data))
        return Y[0] if single else Y


def build_problem(N, L, omegas, g, gdd, psi, mu, V=None, dipole_dir=(0.0, 0.0, 1.0), Rc=None,
                  complex_psi0=False):
    """The setup chain of oracle.bdg_oracle.build_problem through the
    reference's own API: trap (table), wavefunction, contact U_K = U_M = g n,
    dipolar, mu."""
    p = RefProblem(len(N), N, L, complex_psi0)
    p.set_system()
    if V is None:
        from oracle import bdg_oracle as O

        oc = O.Ctx(len(N), N, L, complex_psi0)
        V = O.harmonic_trap(oc, omegas)
    p.set_trap(V)
    p.set_wavefunction(psi)
    p.set_contact(g)
    if gdd != 0.0:
        p.set_dipolar(gdd, dipole_dir, Rc)
    p.set_mu(mu)
    return p
