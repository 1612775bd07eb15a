"""Python bindings of the B200 BdG library (libbdg_b200.so).

Host-side mirror of the reference C API of pstuermer/BDG_LOBPCG
(include/bdg/bdg.h, src/bdg_internal.h): the same functions with the same
argument meaning and error behaviour, bound with ctypes.  All compute runs in
the CUDA library; this module only moves host arrays in and out.  Importing
works without a GPU (for the host-only setup logic); any operator apply or
solve on a machine without a usable GPU fails with the library's error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbdg_b200.so")

# operator codes of include/bdg/bdg_cuda.h
OP_KINETIC, OP_K, OP_M, OP_LREP, OP_SWAP, OP_TK, OP_TM, OP_TLREP, OP_DIPCONV = range(9)
F64, F32 = 0, 1
PREC_F64, PREC_MIXED = 0, 1
CONV_BACKWARD, CONV_TRUE_RESIDUAL = 0, 1
INIT_PLANEWAVE, INIT_WF_WEIGHTED, INIT_REUSE, INIT_CUSTOM = 0, 1, 2, 3
GEOM_AUTO, GEOM_ELONGATED, GEOM_RING = 0, 1, 2
HAS_SYSTEM, HAS_TRAP, HAS_WF, HAS_INTERACTIONS, HAS_DIPOLAR, HAS_MU = (1 << i for i in range(6))

_dp = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)


class MatmulCtx(C.Structure):
    """Layout of matmul_ctx_t (include/bdg/bdg_internal.h)."""

    _fields_ = [
        ("dim", C.c_uint64), ("N", _u64p), ("L", _dp), ("size", C.c_uint64), ("k_size", C.c_uint64),
        ("k2", _dp), ("kx2", C.POINTER(_dp)),
        ("localTermK", _dp), ("localTermM", _dp), ("longRngInt", _dp), ("g_ddi", C.c_double),
        ("mu", C.c_double), ("dipolar", C.c_uint),
        ("wf", C.c_void_p), ("wf_size", C.c_uint64),
        ("fwd_plan", C.c_void_p), ("bwd_plan", C.c_void_p),
        ("f_wrk", C.c_void_p), ("c_wrk1", C.c_void_p), ("c_wrk2", C.c_void_p),
        ("precond_sqrtK", _dp), ("precond_sqrtM", _dp),
        ("complex_psi0", C.c_int),
        ("dev", C.c_void_p), ("prec", C.c_int),
    ]


class SolveStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64), ("refine_iterations", C.c_uint64),
        ("seconds_total", C.c_double), ("seconds_device", C.c_double),
        ("ms_apply_A", C.c_double), ("ms_apply_T", C.c_double), ("ms_residual", C.c_double),
        ("ms_gram", C.c_double), ("ms_small_dense", C.c_double), ("ms_update", C.c_double),
        ("cols_apply_A", C.c_uint64), ("cols_apply_T", C.c_uint64),
        ("max_residual", C.c_double), ("max_true_residual", C.c_double), ("status", C.c_int),
        ("seconds_setup", C.c_double), ("seconds_output", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BdgT(C.Structure):
    """Leading fields of struct bdg_t (include/bdg/bdg_internal.h)."""

    _fields_ = [
        ("ctx", C.POINTER(MatmulCtx)), ("state", C.c_uint32),
        ("nev", C.c_uint64), ("sizeSub", C.c_uint64), ("maxIter", C.c_uint64), ("tol", C.c_double),
        ("complex_psi0", C.c_int),
        ("eigvals", _dp), ("modes_u", C.c_void_p), ("modes_v", C.c_void_p), ("converged", C.c_uint64),
        ("init_mode", C.c_int), ("custom_init_fn", C.c_void_p), ("custom_init_param", C.c_void_p),
        ("reuse_buf", C.c_void_p), ("reuse_n", C.c_uint64), ("reuse_cols", C.c_uint64),
    ]


TRAP_FN = C.CFUNCTYPE(C.c_double, C.c_uint64, _dp, C.c_void_p)
UINT_FN = C.CFUNCTYPE(C.c_double, C.c_void_p, C.c_double)
INIT_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p)

_lib = None


def lib():
    """Load libbdg_b200.so (raises if the library has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} missing: build it with `make -C bdg_lobpcg_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    vp, u64, d, i = C.c_void_p, C.c_uint64, C.c_double, C.c_int
    sig = {
        "bdg_alloc": (vp, [u64, _u64p, _dp, i]),
        "bdg_free": (None, [C.POINTER(vp)]),
        "bdg_reset": (None, [vp]),
        "bdg_set_system": (None, [vp]),
        "bdg_set_trap": (None, [vp, TRAP_FN, vp]),
        "bdg_set_trap_grid": (None, [vp, _dp]),
        "bdg_set_wavefunction": (None, [vp, vp, u64]),
        "bdg_set_local_interactions": (None, [vp, UINT_FN, UINT_FN, vp]),
        "bdg_set_local_interactions_grid": (None, [vp, _dp, _dp]),
        "bdg_set_mu": (None, [vp, d]),
        "bdg_set_dipolar": (None, [vp, d, _dp, d]),
        "bdg_set_solver_params": (None, [vp, u64, u64, u64, d]),
        "bdg_set_init_mode": (None, [vp, i, vp, vp]),
        "bdg_reuse_modes": (i, [vp, d]),
        "bdg_solve": (i, [vp]),
        "bdg_converged": (u64, [vp]),
        "bdg_eigenvalues": (_dp, [vp]),
        "bdg_modes_u": (vp, [vp]),
        "bdg_modes_v": (vp, [vp]),
        "bdg_load_wavefunction": (i, [vp, C.c_char_p]),
        "bdg_write_eigenvalues": (i, [vp, C.c_char_p]),
        "bdg_write_mode_u": (i, [vp, u64, C.c_char_p]),
        "bdg_write_mode_v": (i, [vp, u64, C.c_char_p]),
        "bdg_set_precision": (None, [vp, i]),
        "bdg_set_convergence": (None, [vp, i]),
        "bdg_set_goldstone_deflation": (None, [vp, i]),
        "bdg_set_refinement": (None, [vp, i]),
        "bdg_solve_stats": (C.POINTER(SolveStats), [vp]),
        "bdg_solver_block": (vp, [vp]),
        "matmul_ctx_alloc": (C.POINTER(MatmulCtx), [u64, _u64p, _dp]),
        "matmul_ctx_free": (None, [C.POINTER(C.POINTER(MatmulCtx))]),
        "matmul_ctx_set_system": (None, [C.POINTER(MatmulCtx), i]),
        "dipolar_set_kernel": (None, [C.POINTER(MatmulCtx), d, _dp, d]),
        "dipolar_add_meanfield": (None, [C.POINTER(MatmulCtx)]),
        "bdg_fft_execute": (i, [vp, vp, vp]),
        "bdgd_last_error": (C.c_char_p, []),
        "bdgd_device_count": (i, []),
        "bdgd_create": (i, [C.POINTER(vp), u64, _u64p, _dp, i]),
        "bdgd_destroy": (None, [C.POINTER(vp)]),
        "bdgd_stream": (vp, [vp]),
        "bdgd_synchronize": (i, [vp]),
        "bdgd_set_local_terms": (i, [vp, _dp, _dp]),
        "bdgd_set_wavefunction": (i, [vp, vp]),
        "bdgd_set_precond": (i, [vp, _dp, _dp, d]),
        "bdgd_set_dipolar": (i, [vp, _dp, d, i]),
        "bdgd_apply": (i, [vp, i, i, vp, u64, vp, u64, u64]),
        "bdgd_apply_host": (i, [vp, i, vp, vp, u64]),
        "bdgd_gram": (i, [vp, i, i, u64, u64, vp, u64, vp, u64, vp]),
        "bdgd_block_update": (i, [vp, i, i, u64, u64, i, vp]),
        "bdg_set_initial_block": (i, [vp, vp, u64, u64]),
        "bdg_write_wavefunction_bin": (i, [vp, C.c_char_p]),
        "bdg_write_modes_bin": (i, [vp, i, C.c_char_p]),
        "bdg_write_eigenvalues_bin": (i, [vp, C.c_char_p]),
        "bdg_load_wavefunction_bin": (i, [vp, C.c_char_p]),
        "bdg_lp_create": (i, [C.POINTER(vp), _u64p, i, i, i]),
        "bdg_lp_free": (None, [C.POINTER(vp)]),
        "bdg_lp_nparams": (u64, [vp]),
        "bdg_lp_get_params": (i, [vp, i, vp]),
        "bdg_lp_set_params": (i, [vp, i, vp]),
        "bdg_lp_init_random": (i, [vp, d, u64]),
        "bdg_lp_save": (i, [vp, C.c_char_p]),
        "bdg_lp_load": (i, [vp, C.c_char_p]),
        "bdg_lp_condition": (i, [vp, _dp, _dp, d, d]),
        "bdg_lp_regrid": (i, [vp, _u64p]),
        "bdg_lp_set_energy_loss": (i, [vp, d]),
        "bdg_lp_set_fast_math": (i, [vp, i]),
        "bdg_lp_apply_half": (i, [vp, vp, i, i, vp, u64, vp, u64, u64]),
        "bdg_lp_apply": (i, [vp, vp, i, vp, u64, vp, u64, u64]),
        "bdg_lp_loss_grad": (i, [vp, vp, i, vp, vp, vp, u64, u64, C.POINTER(d), vp]),
        "bdg_lp_train_step": (i, [vp, vp, i, vp, vp, vp, u64, u64, d, C.POINTER(d)]),
        "bdg_lp_cg": (i, [vp, i, d, vp, vp, u64, u64, d, i, C.POINTER(i)]),
        "bdg_set_learned_precond": (i, [vp, vp, i]),
        "bdg_learned_fallback_iteration": (C.c_int64, [vp]),
        "bdg_set_residual_harvest": (i, [vp, vp, u64]),
        "bdg_residual_harvest_count": (u64, [vp]),
        "bdg_device_context": (vp, [vp]),
        "bdg_solve_batch": (i, [C.POINTER(vp), i, i, i, C.POINTER(i), _dp]),
        "bdg_release_device_memory": (None, [vp]),
        "bdgd_set_graphs": (i, [vp, i]),
        "bdgd_fft_tuning": (i, [vp, i, i, C.POINTER(i), C.POINTER(C.c_float)]),
        "bdgd_trim": (i, [vp]),
    }
    for name in ("kinetic", "matmulK", "matmulM", "matmulLrep", "matmulSwap", "precondK", "precondM",
                 "precondLrep", "dipolar_conv"):
        for sfx in ("_d", "_z"):
            sig[name + sfx] = (None, [C.POINTER(MatmulCtx), vp, vp])
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def gpu_available():
    try:
        return lib().bdgd_device_count() > 0
    except Exception:
        return False


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _c_arr(vals, ctype):
    return (ctype * len(vals))(*vals)


# ---------------------------------------------------------------------------
# operator context (reference internal ABI)
# ---------------------------------------------------------------------------
class OperatorContext:
    """matmul_ctx_t with the reference's single-column operators.

    Fields are settable from numpy like the reference tests poke the struct
    (``ctx.localTermK = array`` copies into the C array)."""

    def __init__(self, dim, N, L, complex_psi0=False, set_system=True):
        self._L = lib()
        self.dim = dim
        self.N = list(N)
        self._c = self._L.matmul_ctx_alloc(dim, _c_arr(N, C.c_uint64), _c_arr(L, C.c_double))
        self.cplx = bool(complex_psi0)
        if set_system:
            self._L.matmul_ctx_set_system(self._c, 1 if complex_psi0 else 0)

    def close(self):
        if self._c:
            self._L.matmul_ctx_free(C.byref(self._c))
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def s(self):
        return self._c.contents

    @property
    def size(self):
        return int(self.s.size)

    @property
    def k_size(self):
        return int(self.s.k_size)

    def _arr(self, name, n, dtype=np.float64):
        p = getattr(self.s, name)
        if not p:
            return None
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n * (2 if dtype == np.complex128 else 1),)).view(dtype)

    def get(self, name):
        n = self.k_size if name in ("k2", "longRngInt") else self.size
        if name == "wf":
            return self._arr("wf", self.size, np.complex128 if self.cplx else np.float64)
        return self._arr(name, n)

    def kx2(self, d):
        return np.ctypeslib.as_array(self.s.kx2[d], shape=(self.N[d],))

    def _set_array(self, name, values, dtype=np.float64):
        v = np.ascontiguousarray(values, dtype=dtype).reshape(-1)
        n = self.size
        assert v.size == n, (name, v.size, n)
        cur = getattr(self.s, name)
        nbytes = v.nbytes
        if not cur:
            buf = C.c_void_p(self._alloc(nbytes))
            setattr(self.s, name, C.cast(buf, type(getattr(self.s, name))) if name != "wf" else buf)
            cur = getattr(self.s, name)
        C.memmove(C.cast(cur, C.c_void_p), v.ctypes.data, nbytes)

    def _alloc(self, nbytes):
        libc = C.CDLL(None)
        libc.aligned_alloc.restype = C.c_void_p
        libc.aligned_alloc.argtypes = [C.c_size_t, C.c_size_t]
        p = libc.aligned_alloc(64, (nbytes + 63) // 64 * 64)
        C.memset(p, 0, nbytes)
        return p

    def set(self, name, values):
        if name == "wf":
            self._set_array("wf", values, np.complex128 if self.cplx else np.float64)
            self.s.wf_size = self.size
        else:
            self._set_array(name, values)

    def set_scalar(self, name, v):
        setattr(self.s, name, v)

    def set_dipolar_kernel(self, g_ddi, direction, Rc):
        self._L.dipolar_set_kernel(self._c, g_ddi, _c_arr(direction, C.c_double), Rc)

    def add_meanfield(self):
        self._L.dipolar_add_meanfield(self._c)

    def apply(self, opname, x):
        """Reference single-column operator on a host column (e.g.
        ``apply('matmulK', x)``); the dtype selects _d or _z."""
        x = np.ascontiguousarray(x, dtype=np.complex128 if self.cplx else np.float64)
        y = np.zeros_like(x)
        f = getattr(self._L, opname + ("_z" if self.cplx else "_d"))
        f(self._c, _ptr(x), _ptr(y))
        return y

    def fft(self, forward, x):
        kshape = self.k_size
        if forward:
            x = np.ascontiguousarray(x, dtype=np.complex128 if self.cplx else np.float64)
            out = np.zeros(kshape, dtype=np.complex128)
            plan = self.s.fwd_plan
        else:
            x = np.ascontiguousarray(x, dtype=np.complex128)
            out = np.zeros(self.size, dtype=np.complex128 if self.cplx else np.float64)
            plan = self.s.bwd_plan
        rc = self._L.bdg_fft_execute(plan, _ptr(x), _ptr(out))
        if rc:
            raise RuntimeError(self._L.bdgd_last_error().decode())
        return out


# ---------------------------------------------------------------------------
# problem handle (public API)
# ---------------------------------------------------------------------------
class Problem:
    """bdg_t handle; methods map one-to-one onto include/bdg/bdg.h."""

    def __init__(self, dim, N, L, complex_psi0=False):
        self._L = lib()
        self.dim = dim
        self.N = list(N)
        self.Lbox = list(L)
        self.cplx = bool(complex_psi0)
        self._h = C.c_void_p(self._L.bdg_alloc(dim, _c_arr(N, C.c_uint64), _c_arr(L, C.c_double),
                                               1 if complex_psi0 else 0))
        self._keep = []

    def close(self):
        if self._h:
            self._L.bdg_free(C.byref(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def raw(self):
        return C.cast(self._h, C.POINTER(BdgT)).contents

    @property
    def ctx(self):
        return self.raw.ctx.contents

    @property
    def size(self):
        return int(np.prod(self.N))

    def set_system(self):
        self._L.bdg_set_system(self._h)

    def set_trap(self, V):
        """V: array on the grid, or a callable V(dim, r) (reference callback)."""
        if callable(V):
            cb = TRAP_FN(lambda dim, r, p: float(V(dim, [r[i] for i in range(dim)])))
            self._keep.append(cb)
            self._L.bdg_set_trap(self._h, cb, None)
        else:
            v = np.ascontiguousarray(V, dtype=np.float64).reshape(-1)
            self._L.bdg_set_trap_grid(self._h, _dptr(v))

    def set_wavefunction(self, wf):
        w = np.ascontiguousarray(wf, dtype=np.complex128 if self.cplx else np.float64).reshape(-1)
        self._L.bdg_set_wavefunction(self._h, _ptr(w), w.size)

    def set_local_interactions(self, UK, UM):
        """UK, UM: vectorised callables of the density, evaluated here on
        every grid point and handed to the library as arrays."""
        wf = self.wavefunction()
        n = np.abs(wf) ** 2 if self.cplx else wf * wf
        uK = np.ascontiguousarray(UK(n), dtype=np.float64)
        uM = np.ascontiguousarray(UM(n), dtype=np.float64)
        self._L.bdg_set_local_interactions_grid(self._h, _dptr(uK), _dptr(uM))

    def set_local_interactions_callback(self, UK, UM):
        cK = UINT_FN(lambda p, n: float(UK(n)))
        cM = UINT_FN(lambda p, n: float(UM(n)))
        self._keep += [cK, cM]
        self._L.bdg_set_local_interactions(self._h, cK, cM, None)

    def set_mu(self, mu):
        self._L.bdg_set_mu(self._h, mu)

    def set_dipolar(self, g_ddi, direction, Rc):
        self._L.bdg_set_dipolar(self._h, g_ddi, _c_arr(direction, C.c_double), Rc)

    def set_solver_params(self, nev, sizeSub, maxIter, tol):
        self._L.bdg_set_solver_params(self._h, nev, sizeSub, maxIter, tol)

    def set_init_mode(self, mode, fn=None, param=None):
        if mode == INIT_CUSTOM:
            n, m = 2 * self.size, None

            def cb(bdg, X, n_, m_, p):
                arr = fn(int(n_), int(m_))  # (m, n) block, rows = columns
                arr = np.ascontiguousarray(arr, dtype=np.complex128 if self.cplx else np.float64)
                C.memmove(X, arr.ctypes.data, arr.nbytes)

            c = INIT_FN(cb)
            self._keep.append(c)
            self._L.bdg_set_init_mode(self._h, mode, C.cast(c, C.c_void_p), None)
        else:
            self._L.bdg_set_init_mode(self._h, mode, None, C.c_void_p(param) if param else None)

    def set_initial_block(self, X):
        """Initial block from an (m, n) array (rows = columns of the block; u = v
        for B-positivity), after set_solver_params.  The library borrows the
        array (bdg_set_initial_block); this object keeps it alive."""
        X = np.ascontiguousarray(X, dtype=np.complex128 if self.cplx else np.float64)
        m, n = X.shape
        rc = self._L.bdg_set_initial_block(self._h, C.c_void_p(X.ctypes.data), n, m)
        if rc:
            raise ValueError(f"bdg_set_initial_block: block {m} x {n} does not fit the problem ({rc})")
        self._x0 = X

    def reuse_modes(self, noise_frac):
        return self._L.bdg_reuse_modes(self._h, noise_frac)

    def set_precision(self, p):
        self._L.bdg_set_precision(self._h, p)

    def set_convergence(self, c):
        self._L.bdg_set_convergence(self._h, c)

    def set_goldstone_deflation(self, on):
        self._L.bdg_set_goldstone_deflation(self._h, 1 if on else 0)

    def set_learned_precond(self, lp, stall_window=0):
        rc = self._L.bdg_set_learned_precond(self._h, lp._p if lp is not None else None, stall_window)
        if rc:
            raise RuntimeError(f"bdg_set_learned_precond failed ({rc})")
        self._keep.append(lp)

    def learned_fallback_iteration(self):
        return int(self._L.bdg_learned_fallback_iteration(self._h))

    def set_residual_harvest(self, ptr, cap_cols):
        self._L.bdg_set_residual_harvest(self._h, C.c_void_p(ptr) if ptr else None, cap_cols)

    def residual_harvest_count(self):
        return int(self._L.bdg_residual_harvest_count(self._h))

    def device_context(self):
        """The problem's own device context (operators uploaded), borrowed."""
        p = self._L.bdg_device_context(self._h)
        if not p:
            raise RuntimeError("bdg_device_context failed: " + self._L.bdgd_last_error().decode())
        return DeviceContext.borrow(p, self.size, self.cplx)

    def set_refinement(self, n):
        self._L.bdg_set_refinement(self._h, n)

    def solve(self):
        return int(self._L.bdg_solve(self._h))

    def converged(self):
        return int(self._L.bdg_converged(self._h))

    def eigenvalues(self):
        p = self._L.bdg_eigenvalues(self._h)
        if not p:
            return None
        return np.ctypeslib.as_array(p, shape=(int(self.raw.nev),)).copy()

    def _modes(self, fn):
        p = fn(self._h)
        if not p:
            return None
        nev = int(self.raw.nev)
        dt = np.complex128 if self.cplx else np.float64
        n = self.size * nev * (2 if self.cplx else 1)
        a = np.ctypeslib.as_array(C.cast(p, _dp), shape=(n,)).copy().view(dt)
        return a.reshape(nev, self.size)

    def modes_u(self):
        return self._modes(self._L.bdg_modes_u)

    def modes_v(self):
        return self._modes(self._L.bdg_modes_v)

    def block(self):
        p = self._L.bdg_solver_block(self._h)
        if not p:
            return None
        m = int(self.raw.sizeSub)
        n = 2 * self.size
        cnt = n * m * (2 if self.cplx else 1)
        a = np.ctypeslib.as_array(C.cast(p, _dp), shape=(cnt,)).copy()
        return a.view(np.complex128 if self.cplx else np.float64).reshape(m, n)

    def stats(self):
        return self._L.bdg_solve_stats(self._h).contents.as_dict()

    def wavefunction(self):
        c = self.ctx
        if not c.wf:
            return None
        n = self.size * (2 if self.cplx else 1)
        a = np.ctypeslib.as_array(C.cast(c.wf, _dp), shape=(n,)).copy()
        return a.view(np.complex128) if self.cplx else a

    def local_terms(self):
        c = self.ctx
        K = np.ctypeslib.as_array(c.localTermK, shape=(self.size,)).copy()
        M = np.ctypeslib.as_array(c.localTermM, shape=(self.size,)).copy()
        return K, M

    def state(self):
        return int(self.raw.state)

    def write_eigenvalues(self, fn):
        return self._L.bdg_write_eigenvalues(self._h, fn.encode())

    def write_mode_u(self, idx, base):
        return self._L.bdg_write_mode_u(self._h, idx, base.encode())

    def write_mode_v(self, idx, base):
        return self._L.bdg_write_mode_v(self._h, idx, base.encode())

    def load_wavefunction(self, fn):
        return self._L.bdg_load_wavefunction(self._h, fn.encode())

    # binary files (read them with bdg_lobpcg_b200.binio.read)
    def write_wavefunction_bin(self, fn):
        return self._L.bdg_write_wavefunction_bin(self._h, fn.encode())

    def write_modes_bin(self, part, fn):
        """part 0: u, 1: v (all nev modes)."""
        return self._L.bdg_write_modes_bin(self._h, part, fn.encode())

    def write_eigenvalues_bin(self, fn):
        return self._L.bdg_write_eigenvalues_bin(self._h, fn.encode())

    def load_wavefunction_bin(self, fn):
        return self._L.bdg_load_wavefunction_bin(self._h, fn.encode())


# ---------------------------------------------------------------------------
# device context (block entry points on device pointers)
# ---------------------------------------------------------------------------
class _UpdateTerm(C.Structure):
    _fields_ = [("s", C.c_void_p), ("c", C.c_void_p), ("k", C.c_int), ("ldc", C.c_int)]


class _UpdateOut(C.Structure):
    _fields_ = [("y", C.c_void_p), ("ncol", C.c_int), ("nterm", C.c_int), ("alpha", C.c_double),
                ("beta", C.c_double), ("term", _UpdateTerm * 3)]


class DeviceContext:
    """bdgd_ctx: batched operator applies on device memory (bdg_cuda.h)."""

    @classmethod
    def borrow(cls, ptr, size, complex_psi0=False):
        """Wrap a context owned by the library (e.g. bdg_device_context)."""
        self = cls.__new__(cls)
        self._L = lib()
        self._c = C.c_void_p(ptr)
        self._owned = False
        self.cplx = bool(complex_psi0)
        self.size = int(size)
        return self

    def __init__(self, dim, N, L, complex_psi0=False):
        self._L = lib()
        self._owned = True
        self._c = C.c_void_p()
        rc = self._L.bdgd_create(C.byref(self._c), dim, _c_arr(N, C.c_uint64), _c_arr(L, C.c_double),
                                 1 if complex_psi0 else 0)
        self.check(rc)
        self.cplx = bool(complex_psi0)
        self.size = int(np.prod(N))

    def check(self, rc):
        if rc:
            raise RuntimeError(f"bdgd error {rc}: {self._L.bdgd_last_error().decode()}")

    def close(self):
        if self._c and getattr(self, "_owned", True):
            self._L.bdgd_destroy(C.byref(self._c))
        self._c = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ptr(self):
        return self._c.value

    @property
    def stream(self):
        return self._L.bdgd_stream(self._c)

    def set_fields(self, ltK=None, ltM=None, wf=None, pK=None, pM=None, mu=0.0, vdd=None, g_ddi=0.0, dipolar=False):
        L = self._L
        f = lambda a: _dptr(np.ascontiguousarray(a, dtype=np.float64)) if a is not None else None
        keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (ltK, ltM, pK, pM, vdd)]
        self.check(L.bdgd_set_local_terms(self._c, *(_dptr(k) if k is not None else None for k in keep[:2])))
        if wf is not None:
            w = np.ascontiguousarray(wf, dtype=np.complex128 if self.cplx else np.float64)
            self.check(L.bdgd_set_wavefunction(self._c, _ptr(w)))
        if keep[2] is not None:
            self.check(L.bdgd_set_precond(self._c, _dptr(keep[2]), _dptr(keep[3]), mu))
        self.check(L.bdgd_set_dipolar(self._c, _dptr(keep[4]) if keep[4] is not None else None, g_ddi,
                                      1 if dipolar else 0))

    def apply_ptr(self, op, prec, x_ptr, ldx, y_ptr, ldy, ncol):
        self.check(self._L.bdgd_apply(self._c, op, prec, C.c_void_p(x_ptr), ldx, C.c_void_p(y_ptr), ldy, ncol))

    def apply_host(self, op, X):
        X = np.ascontiguousarray(X)
        Y = np.zeros_like(X)
        ncol = X.shape[0] if X.ndim == 2 else 1
        self.check(self._L.bdgd_apply_host(self._c, op, _ptr(X), _ptr(Y), ncol))
        return Y

    def gram_ptr(self, prec, cplx, half, k, S_ptr, lds, AS_ptr, ldas, out_ptr):
        self.check(self._L.bdgd_gram(self._c, prec, 1 if cplx else 0, half, k, C.c_void_p(S_ptr), lds,
                                     C.c_void_p(AS_ptr), ldas, C.c_void_p(out_ptr)))

    def block_update(self, prec, cplx, n, ld, outs):
        """bdgd_block_update: outs = [(y_ptr, ncol, alpha, beta, [(s_ptr, k, c_ptr, ldc), ...]), ...].
        Returns the library's status (BDGD_ERR_UNSUPPORTED = -3 launches nothing)."""
        arr = (_UpdateOut * len(outs))()
        for o, (y, ncol, alpha, beta, terms) in zip(arr, outs):
            o.y, o.ncol, o.nterm, o.alpha, o.beta = y, ncol, len(terms), alpha, beta
            for t, (sp, k, cp, ldc) in zip(o.term, terms):
                t.s, t.k, t.c, t.ldc = sp, k, cp, ldc
        return self._L.bdgd_block_update(self._c, prec, 1 if cplx else 0, n, ld, len(outs),
                                         C.cast(arr, C.c_void_p))

    def synchronize(self):
        self.check(self._L.bdgd_synchronize(self._c))

    def set_graphs(self, on):
        self.check(self._L.bdgd_set_graphs(self._c, 1 if on else 0))

    def fft_tuning(self, op, prec):
        """(path, [ms_reg, ms_ct]) chosen by the autotuner; path 0 = not tuned."""
        path = C.c_int()
        ms = (C.c_float * 2)()
        self.check(self._L.bdgd_fft_tuning(self._c, op, prec, C.byref(path), ms))
        return path.value, [ms[0], ms[1]]


# ---------------------------------------------------------------------------
# learned SPD preconditioner (bdg/bdg_learn.h)
# ---------------------------------------------------------------------------
class LearnedPrecond:
    """bdg_lp: T = S^T S + exp(eta) P0 per half; see include/bdg/bdg_learn.h."""

    HALF_K, HALF_M = 0, 1

    def __init__(self, N, C_=16, L=4, modes=12):
        self._L = lib()
        self._p = C.c_void_p()
        self.N = list(N)
        self.shape = (C_, L, modes)
        self._check(self._L.bdg_lp_create(C.byref(self._p), _c_arr(N, C.c_uint64), C_, L, modes))

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"bdg_lp error {rc}: {self._L.bdgd_last_error().decode()}")

    def close(self):
        if self._p:
            self._L.bdg_lp_free(C.byref(self._p))
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nparams(self):
        return int(self._L.bdg_lp_nparams(self._p))

    def get_params(self, half):
        a = np.zeros(self.nparams, dtype=np.float32)
        self._check(self._L.bdg_lp_get_params(self._p, half, _ptr(a)))
        return a

    def set_params(self, half, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        self._check(self._L.bdg_lp_set_params(self._p, half, _ptr(a)))

    def init_random(self, amp, seed):
        self._check(self._L.bdg_lp_init_random(self._p, amp, seed))

    def save(self, path):
        self._check(self._L.bdg_lp_save(self._p, str(path).encode()))

    def load(self, path):
        self._check(self._L.bdg_lp_load(self._p, str(path).encode()))

    def condition(self, psi0, V, eps_dd, lam):
        psi0 = np.ascontiguousarray(psi0, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        self._check(self._L.bdg_lp_condition(self._p, _dptr(psi0), _dptr(V), eps_dd, lam))

    def set_fast_math(self, on):
        """Applies with TF32 tensor-core basis GEMMs (default) or exact FP32."""
        self._check(self._L.bdg_lp_set_fast_math(self._p, 1 if on else 0))

    def set_energy_loss(self, sigma):
        """sigma >= 0: energy-norm loss of A = Op + sigma; sigma < 0: L2 loss."""
        self._check(self._L.bdg_lp_set_energy_loss(self._p, sigma))

    def regrid(self, N):
        self.N = list(N)
        self._check(self._L.bdg_lp_regrid(self._p, _c_arr(N, C.c_uint64)))

    def apply_half_ptr(self, dev, half, prec, x_ptr, ldx, y_ptr, ldy, ncol):
        self._check(self._L.bdg_lp_apply_half(self._p, C.c_void_p(dev.ptr), half, prec, C.c_void_p(x_ptr), ldx,
                                              C.c_void_p(y_ptr), ldy, ncol))

    def apply_ptr(self, dev, prec, x_ptr, ldx, y_ptr, ldy, ncol):
        self._check(self._L.bdg_lp_apply(self._p, C.c_void_p(dev.ptr), prec, C.c_void_p(x_ptr), ldx,
                                         C.c_void_p(y_ptr), ldy, ncol))

    def loss_grad(self, dev, half, r_ptr, e_ptr, p0r_ptr, ld, ncol, want_grad=True):
        loss = C.c_double()
        g = np.zeros(self.nparams, dtype=np.float32) if want_grad else None
        self._check(self._L.bdg_lp_loss_grad(self._p, C.c_void_p(dev.ptr), half, C.c_void_p(r_ptr),
                                             C.c_void_p(e_ptr), C.c_void_p(p0r_ptr), ld, ncol, C.byref(loss),
                                             _ptr(g) if want_grad else None))
        return loss.value, g

    def train_step(self, dev, half, r_ptr, e_ptr, p0r_ptr, ld, ncol, lr):
        loss = C.c_double()
        self._check(self._L.bdg_lp_train_step(self._p, C.c_void_p(dev.ptr), half, C.c_void_p(r_ptr),
                                              C.c_void_p(e_ptr), C.c_void_p(p0r_ptr), ld, ncol, lr,
                                              C.byref(loss)))
        return loss.value


def lp_cg(dev, op, sigma, r_ptr, e_ptr, ld, ncol, tol, maxit):
    """e = (op + sigma)^-1 r on device columns (bdg_lp_cg); returns iterations."""
    it = C.c_int()
    rc = lib().bdg_lp_cg(C.c_void_p(dev.ptr), op, sigma, C.c_void_p(r_ptr), C.c_void_p(e_ptr), ld, ncol, tol,
                         maxit, C.byref(it))
    if rc:
        raise RuntimeError(f"bdg_lp_cg error {rc}: {lib().bdgd_last_error().decode()}")
    return it.value


def solve_batch(problems, concurrency=8, graphs=True):
    """bdg_solve_batch over Problem objects; returns (return codes, seconds)."""
    n = len(problems)
    arr = (C.c_void_p * n)(*[p._h.value for p in problems])
    rcs = (C.c_int * n)()
    secs = np.zeros(n)
    lib().bdg_solve_batch(arr, n, concurrency, 1 if graphs else 0, rcs, _dptr(secs))
    return [rcs[i] for i in range(n)], secs
