"""Synthetic dipolar-trap BdG problems (the benchmark configurations).

A problem is the dimensionless dipolar GPE of a harmonic trap
(1, 1, lambda) in a periodic box, contact coupling g, dipolar coupling
g_dd = eps_dd * g along z with a spherical cutoff R_c, and its stationary
ground state psi0 from the library's GPU producer (split-step imaginary time
until |d mu| < 1e-12, then bordered Newton polish).  `build` sets the BdG
problem up through the public API (trap, wavefunction, contact callbacks
U_K = U_M = g n, dipolar kernel, mu), with the true-residual criterion,
Goldstone deflation and an initial block X0 ~ N(0, 1) with v = u.
"""
import ctypes as C

import numpy as np


def config(grid, eps_dd=None, lam=2.0, g=1000.0, nev=None, seed=None, box=None):
    """Benchmark configuration: 32^3 in [-8, 8)^3 (eps_dd 0.5, nev 8, seed 0)
    or 64^3 / 128^3 in [-12, 12)^3 (eps_dd 0.7, nev 16 / 32, seed 1)."""
    if nev is None:
        nev = {32: 8, 64: 16, 128: 32}.get(grid, 32)
    if box is None:
        box = 16.0 if grid == 32 else 24.0
    if eps_dd is None:
        eps_dd = 0.5 if grid == 32 else 0.7
    if seed is None:
        seed = 0 if grid == 32 else 1
    return dict(N=[grid] * 3, L=[box] * 3, omegas=(1.0, 1.0, lam), g=g, gdd=g * eps_dd, eps_dd=eps_dd, lam=lam,
                rc=8.0, nev=nev, sizeSub=2 * nev, tol=1e-8, seed=seed)


def grid_coords(N, L):
    """x_i = (i - N/2) L / N per axis (the reference's grid, src/setup.c:17-84)."""
    return [(np.arange(n) - 0.5 * n) * l / n for n, l in zip(N, L)]


def trap(N, L, om):
    x, y, z = grid_coords(N, L)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return (0.5 * (om[0] ** 2 * X ** 2 + om[1] ** 2 * Y ** 2 + om[2] ** 2 * Z ** 2)).reshape(-1)


def ground_state(B, cfg, max_steps=200000):
    """Stationary psi0 on the GPU (bdg_ground_state); returns psi, mu,
    imaginary-time steps, stationarity ||H psi - mu psi|| and the trap V."""
    N, L = cfg["N"], cfg["L"]
    x, y, z = grid_coords(N, L)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    psi = np.exp(-0.5 * (X * X + Y * Y + Z * Z)).reshape(-1).copy()
    V = trap(N, L, cfg["omegas"])
    lib = B.lib()
    f = lib.bdg_ground_state
    f.restype = C.c_int
    f.argtypes = [C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_void_p, C.c_double, C.c_double,
                  C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_void_p,
                  C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    mu = C.c_double()
    steps = C.c_uint64()
    stat = C.c_double()
    rc = f(3, (C.c_uint64 * 3)(*N), (C.c_double * 3)(*L), V.ctypes.data, cfg["g"], cfg["gdd"],
           (C.c_double * 3)(0.0, 0.0, 1.0), cfg["rc"], 1e-3, 1e-12, max_steps, 4, psi.ctypes.data, C.byref(mu),
           C.byref(steps), C.byref(stat))
    if rc:
        raise RuntimeError(f"bdg_ground_state failed ({rc})")
    return psi, mu.value, int(steps.value), stat.value, V


def build(B, cfg, psi, mu, V, precision="f64", maxiter=2000):
    """The BdG problem through the public API; returns (Problem, X0)."""
    p = B.Problem(3, cfg["N"], cfg["L"])
    p.set_system()
    p.set_trap(V)
    p.set_wavefunction(psi)
    g = cfg["g"]
    p.set_local_interactions(lambda n: g * n, lambda n: g * n)
    p.set_dipolar(cfg["gdd"], [0.0, 0.0, 1.0], cfg["rc"])
    p.set_mu(mu)
    p.set_solver_params(cfg["nev"], cfg["sizeSub"], maxiter, cfg["tol"])
    p.set_convergence(B.CONV_TRUE_RESIDUAL)
    p.set_goldstone_deflation(True)
    p.set_precision(B.PREC_MIXED if precision == "mixed" else B.PREC_F64)
    size = int(np.prod(cfg["N"]))
    rng = np.random.default_rng(cfg["seed"])
    u = rng.standard_normal((cfg["sizeSub"], size))
    X0 = np.concatenate([u, u], axis=1)
    p.set_initial_block(X0)
    return p, X0
