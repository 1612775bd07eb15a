"""CPU FP64 oracle for the BdG operator-and-solver path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product library imports, links or
calls this module: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it, and only as the checker / the timed CPU
baseline.

It restates, in numpy/scipy, the algorithm of the reference library
pstuermer/BDG_LOBPCG for the operator path (file:line citations below are
relative to that project's root):

* k-space tables              src/matmul_ctx.c:88-132
* kinetic  y = F^-1[k^2/2 F x] src/kinetic_impl.inc:17-30
* K        kinetic + ltK x     src/matmulK_impl.inc:11-28
* M        kinetic + ltM x + 2 dipolar_conv(x)   src/matmulM_impl.inc:14-44
* dipolar exchange convolution src/dipolar_conv_impl.inc:22-52
* Lrep = [K u; M v]            src/matmulLrep_impl.inc:13-18
* Swap = [x_v; x_u]            src/matmulSwap_impl.inc:14-26
* preconditioner T_K, T_M, T_Lrep   src/precond_impl.inc:21-118
* dipolar kernel / mean field  src/dipolar.c:21-72, src/dipolar_meanfield_impl.inc:20-55
* setup (trap grid, interactions, mu, precond sqrt)   src/setup.c:17-197
* init modes: PLANEWAVE (real and complex), complex WF_WEIGHTED
                                                      src/solver.c:68-259, :321-414

FFTs follow FFTW's conventions as the reference uses them: unnormalised
transforms, dims reversed so x is fastest, r2c halving the x axis
(src/matmul_ctx.c:149-169).

The eigensolver the reference links (``d_ilobpcg``/``z_ilobpcg`` from an
external, unvendored "LOBPCG" library, call sites src/solver.c:147-164,
262-283) is restated from the published method: Kressner, Miloloza Pandur &
Shao, "An indefinite variant of LOBPCG for definite matrix pencils",
Numer. Algorithms 66 (2014) -- block trace minimisation of x^T A x / x^T B x
over B-positive subspaces, Rayleigh-Ritz on span[X, T R, P].  The GPU solver
in the product runs the same iteration; see ``ilobpcg`` below.

Parity pinning (tests/test_ref_oracle_cpu.py, tests/test_oracle_cpu.py):
* against the reference's own C sources, compiled unmodified into
  oracle/_ref (oracle/Makefile): setup fields and all nine operators to
  1e-13 on the 32^3 benchmark trap (real and complex psi0), the init-mode
  blocks bit for bit (real) or to the rounding of cabs (complex), and the
  solve of the reference's own solve path on the same inputs;
* the reference's own tests/test_*.c, run against that build;
* the known-answer assertions of those tests, restated in tests/cases.py.
"""
from __future__ import annotations

import math
import os

import numpy as np
import scipy.fft as sfft
import scipy.linalg as sla

_WORKERS = int(os.environ.get("BDG_ORACLE_THREADS", os.cpu_count() or 1))

BDG_INIT_PLANEWAVE, BDG_INIT_WF_WEIGHTED, BDG_INIT_REUSE, BDG_INIT_CUSTOM = 0, 1, 2, 3
BDG_GEOM_AUTO, BDG_GEOM_ELONGATED, BDG_GEOM_RING = 0, 1, 2


# ----------------------------------------------------------------------------
# context
# ----------------------------------------------------------------------------
class Ctx:
    """Field-for-field analogue of the reference ``matmul_ctx_t``
    (src/bdg_internal.h:71-115)."""

    def __init__(self, dim, N, L, complex_psi0=False):
        self.dim = int(dim)
        self.N = [int(n) for n in N][:dim]
        self.L = [float(l) for l in L][:dim]
        self.size = int(np.prod(self.N))
        self.complex_psi0 = bool(complex_psi0)
        self.k_size = 0
        self.k2 = None
        self.kx2 = None
        self.localTermK = np.zeros(self.size)
        self.localTermM = np.zeros(self.size)
        self.longRngInt = None
        self.g_ddi = 0.0
        self.mu = 0.0
        self.dipolar = False
        self.wf = None
        self.precond_sqrtK = None
        self.precond_sqrtM = None

    # shape of a real-space field in C order: (Nz, Ny, Nx)
    @property
    def rshape(self):
        return tuple(reversed(self.N))

    @property
    def kshape(self):
        s = list(self.rshape)
        if not self.complex_psi0:
            s[-1] = self.N[0] // 2 + 1
        return tuple(s)

    @property
    def ctype(self):
        return np.complex128 if self.complex_psi0 else np.float64


def set_system(ctx: Ctx):
    """k tables exactly as src/matmul_ctx.c:88-132 builds them."""
    N = ctx.N
    if ctx.complex_psi0:
        ctx.k_size = ctx.size
    else:
        ctx.k_size = (N[0] // 2 + 1) * int(np.prod(N[1:]))
    ctx.kx2 = []
    for d in range(ctx.dim):
        dk = 2.0 * math.pi / ctx.L[d]
        j = np.arange(N[d])
        kj = np.where(j <= N[d] // 2, dk * j, dk * (j - N[d]))
        ctx.kx2.append(kj * kj)
    n0k = N[0] if ctx.complex_psi0 else N[0] // 2 + 1
    k2 = ctx.kx2[0][:n0k].copy()
    # summation order of the reference: kx2[0][ix] + kx2[1][iy] + kx2[2][iz]
    if ctx.dim >= 2:
        k2 = k2[None, :] + ctx.kx2[1][:, None]
    if ctx.dim == 3:
        k2 = k2[None, :, :] + ctx.kx2[2][:, None, None]
    ctx.k2 = np.ascontiguousarray(k2).reshape(-1)
    return ctx


# ----------------------------------------------------------------------------
# unnormalised FFTs on blocks shaped (ncol, *rshape)
# ----------------------------------------------------------------------------
def _axes(ctx):
    return tuple(range(1, ctx.dim + 1))


def fft_fwd(ctx, x):
    x = x.reshape((-1,) + ctx.rshape)
    if ctx.complex_psi0:
        return sfft.fftn(x, axes=_axes(ctx), workers=_WORKERS)
    return sfft.rfftn(x, axes=_axes(ctx), workers=_WORKERS)


def fft_bwd(ctx, X):
    # unnormalised inverse (FFTW_BACKWARD / c2r)
    if ctx.complex_psi0:
        y = sfft.ifftn(X, axes=_axes(ctx), norm="forward", workers=_WORKERS)
    else:
        y = sfft.irfftn(X, s=ctx.rshape, axes=_axes(ctx), norm="forward", workers=_WORKERS)
    return y.reshape(y.shape[0], -1)


def _blk(x, ctx):
    x = np.asarray(x)
    single = x.ndim == 1
    return (x.reshape(1, -1) if single else x), single


def _out(y, single):
    return y[0] if single else y


def _k(ctx, a):
    return a.reshape(ctx.kshape)


# ----------------------------------------------------------------------------
# operators (single column: shape (size,), block: shape (ncol, size))
# ----------------------------------------------------------------------------
def kinetic(ctx, x):
    """src/kinetic_impl.inc:17-30: fk *= k2 * (0.5/size)."""
    x, s = _blk(x, ctx)
    fk = fft_fwd(ctx, x)
    fk *= _k(ctx, ctx.k2 * (0.5 / ctx.size))
    return _out(fft_bwd(ctx, fk), s)


def matmulK(ctx, x):
    """src/matmulK_impl.inc:11-28: y = kinetic(x) + ltK*x."""
    x, s = _blk(x, ctx)
    y = kinetic(ctx, x)
    y = y + ctx.localTermK[None, :] * x
    return _out(y, s)


def dipolar_conv(ctx, v):
    """src/dipolar_conv_impl.inc:22-52: g*wf*F^-1[kernel/size * F(conj(wf)*v)]."""
    v, s = _blk(v, ctx)
    wf = ctx.wf
    buf = (np.conj(wf) if ctx.complex_psi0 else wf)[None, :] * v
    fk = fft_fwd(ctx, buf)
    fk *= _k(ctx, ctx.longRngInt * (1.0 / ctx.size))
    buf = fft_bwd(ctx, fk)
    out = (ctx.g_ddi * wf)[None, :] * buf
    return _out(out, s)


def matmulM(ctx, x):
    """src/matmulM_impl.inc:14-44."""
    x, s = _blk(x, ctx)
    y = kinetic(ctx, x)
    if ctx.dipolar and ctx.dim == 3:
        dc = dipolar_conv(ctx, x)
        y = y + (ctx.localTermM[None, :] * x + 2.0 * dc)
    else:
        y = y + ctx.localTermM[None, :] * x
    return _out(y, s)


def matmulLrep(ctx, x):
    """src/matmulLrep_impl.inc:13-18: [K u; M v]."""
    x, s = _blk(x, ctx)
    S = ctx.size
    y = np.empty_like(x, dtype=np.result_type(x, np.float64))
    y[:, :S] = matmulK(ctx, x[:, :S])
    y[:, S:] = matmulM(ctx, x[:, S:])
    return _out(y, s)


def matmulSwap(ctx, x):
    """src/matmulSwap_impl.inc:14-26."""
    x, s = _blk(x, ctx)
    S = ctx.size
    y = np.concatenate([x[:, S:], x[:, :S]], axis=1)
    return _out(y, s)


def safe_val(x):
    """src/bdg_internal.h:47-50."""
    return np.where(np.abs(x) < 1e-8, 1e-8, x)


def _precond(ctx, p, x):
    """src/precond_impl.inc:21-65 (T_K) and :67-111 (T_M)."""
    x, s = _blk(x, ctx)
    buf = p[None, :] * x
    fk = fft_fwd(ctx, buf)
    fk *= _k(ctx, (1.0 / ctx.size) / safe_val(ctx.mu + 0.5 * ctx.k2))
    y = fft_bwd(ctx, fk)
    y = y * p[None, :]
    return _out(y, s)


def precondK(ctx, x):
    return _precond(ctx, ctx.precond_sqrtK, x)


def precondM(ctx, x):
    return _precond(ctx, ctx.precond_sqrtM, x)


def precondLrep(ctx, x):
    """src/precond_impl.inc:113-118."""
    x, s = _blk(x, ctx)
    S = ctx.size
    y = np.empty_like(x, dtype=np.result_type(x, np.float64))
    y[:, :S] = precondK(ctx, x[:, :S])
    y[:, S:] = precondM(ctx, x[:, S:])
    return _out(y, s)


# ----------------------------------------------------------------------------
# dipolar kernel and mean field
# ----------------------------------------------------------------------------
def dipolar_set_kernel(ctx, g_ddi, dipole_dir, cutoff_radius):
    """src/dipolar.c:21-72: (3 cos^2 theta - 1) * C(kR), kernel(k=0) = 0."""
    ctx.g_ddi = float(g_ddi)
    Nx, Ny, Nz = ctx.N
    n0k = Nx if ctx.complex_psi0 else Nx // 2 + 1
    dkx, dky, dkz = (2.0 * math.pi / l for l in ctx.L)
    ix = np.arange(n0k)
    fx = np.where(ctx.complex_psi0 & (ix > Nx // 2), ix - Nx, ix)
    iy = np.arange(Ny)
    fy = np.where(iy <= Ny // 2, iy, iy - Ny)
    iz = np.arange(Nz)
    fz = np.where(iz <= Nz // 2, iz, iz - Nz)
    kx = (dkx * fx)[None, None, :]
    ky = (dky * fy)[None, :, None]
    kz = (dkz * fz)[:, None, None]
    ksq = kx * kx + ky * ky + kz * kz
    d = np.asarray(dipole_dir, dtype=np.float64)
    dir_sq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
    kdotd = kx * d[0] + ky * d[1] + kz * d[2]
    with np.errstate(divide="ignore", invalid="ignore"):
        cos_sq = (kdotd * kdotd) / (ksq * dir_sq)
        kmag = np.sqrt(ksq)
        kR = kmag * cutoff_radius
        kR2 = kR * kR
        fcut = 1.0 + 3.0 * np.cos(kR) / kR2 - 3.0 * np.sin(kR) / (kR2 * kR)
        ker = (3.0 * cos_sq - 1.0) * fcut
    ker = np.where(ksq < 1e-50, 0.0, ker)
    ctx.longRngInt = np.ascontiguousarray(ker).reshape(-1)
    return ctx.longRngInt


def dipolar_add_meanfield(ctx):
    """src/dipolar_meanfield_impl.inc:20-55."""
    wf = ctx.wf
    dens = (np.abs(wf) ** 2).astype(ctx.ctype)
    fk = fft_fwd(ctx, dens[None, :])
    fk *= _k(ctx, ctx.longRngInt * (1.0 / ctx.size))
    buf = fft_bwd(ctx, fk)[0]
    phi = ctx.g_ddi * np.real(buf)
    ctx.localTermK = ctx.localTermK + phi
    ctx.localTermM = ctx.localTermM + phi


# ----------------------------------------------------------------------------
# physics setup (src/setup.c)
# ----------------------------------------------------------------------------
def grid_coords(ctx):
    """x_i = (i - N/2) L / N per axis (src/setup.c:35, :68-72)."""
    return [((np.arange(n) - 0.5 * n) * l / n) for n, l in zip(ctx.N, ctx.L)]


def set_trap_array(ctx, V):
    """src/setup.c:17-84 with the callback already evaluated on the grid."""
    V = np.asarray(V, dtype=np.float64).reshape(-1)
    ctx.localTermK = ctx.localTermK + V
    ctx.localTermM = ctx.localTermM + V


def harmonic_trap(ctx, omegas):
    c = grid_coords(ctx)
    mesh = np.meshgrid(*reversed(c), indexing="ij")  # (z, y, x) order
    mesh = list(reversed(mesh))  # x, y, z
    V = np.zeros(ctx.rshape)
    for d in range(ctx.dim):
        V = V + 0.5 * omegas[d] ** 2 * mesh[d] ** 2
    return V.reshape(-1)


def set_wavefunction(ctx, wf):
    """src/setup.c:89-114 (copies)."""
    ctx.wf = np.array(wf, dtype=ctx.ctype).reshape(-1).copy()


def set_local_interactions(ctx, UK, UM):
    """src/setup.c:119-145 with vectorised callbacks UK(n), UM(n)."""
    dens = np.abs(ctx.wf) ** 2 if ctx.complex_psi0 else ctx.wf * ctx.wf
    uK = UK(dens)
    uM = UM(dens)
    ctx.localTermK = ctx.localTermK + uK
    ctx.localTermM = ctx.localTermM + (uK + 2.0 * uM)


def set_mu(ctx, mu):
    """src/setup.c:150-177: precond sqrt arrays before subtracting mu."""
    ctx.precond_sqrtK = 1.0 / np.sqrt(np.fmax(1e-8, ctx.localTermK))
    ctx.precond_sqrtM = 1.0 / np.sqrt(np.fmax(1e-8, ctx.localTermM))
    ctx.localTermK = ctx.localTermK - mu
    ctx.localTermM = ctx.localTermM - mu
    ctx.mu = float(mu)


def set_dipolar(ctx, g_ddi, dipole_dir, cutoff_radius):
    """src/setup.c:182-197."""
    if ctx.dim != 3:
        raise ValueError("dipolar interactions require dim == 3")
    dipolar_set_kernel(ctx, g_ddi, dipole_dir, cutoff_radius)
    dipolar_add_meanfield(ctx)
    ctx.dipolar = True


# ----------------------------------------------------------------------------
# PRNG helpers of the reference (src/bdg_internal.h:52-65)
# ----------------------------------------------------------------------------
class XorShift32:
    def __init__(self, seed):
        self.s = np.uint32(seed)

    def next(self):
        x = int(self.s)
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        self.s = np.uint32(x)
        return x

    def xrand(self):
        return float(self.next() & 0x7FFFFFFF) / float(0x7FFFFFFF)

    def xrand_many(self, count):
        out = np.empty(count)
        for i in range(count):
            out[i] = self.xrand()
        return out


# ----------------------------------------------------------------------------
# init modes (src/solver.c:68-259)
# ----------------------------------------------------------------------------
def enumerate_kvecs(ctx, hint, n_needed):
    """src/solver.c:76-129 (stable sort on |k|^2 as qsort does with ties
    broken by enumeration order only when the sort is stable; the reference
    uses qsort, so tie order among equal |k|^2 is implementation-defined)."""
    dim = ctx.dim
    rng = [1, 1, 1]
    if hint == BDG_GEOM_ELONGATED:
        long_d = 0
        for d in range(1, dim):
            if ctx.L[d] > ctx.L[long_d]:
                long_d = d
        rng[long_d] = min(ctx.N[long_d], 2 * n_needed)
    elif hint == BDG_GEOM_RING:
        for d in range(min(dim, 2)):
            rng[d] = min(ctx.N[d], 2 * n_needed)
    else:
        for d in range(dim):
            rng[d] = min(ctx.N[d], 2 * n_needed)
    ent = []
    for iz in range(rng[2]):
        kz2 = ctx.kx2[2][iz] if dim > 2 else 0.0
        for iy in range(rng[1]):
            ky2 = ctx.kx2[1][iy] if dim > 1 else 0.0
            for ix in range(rng[0]):
                ent.append((ctx.kx2[0][ix] + ky2 + kz2, (ix, iy, iz)))
    ent.sort(key=lambda e: e[0])
    return ent, min(len(ent), n_needed)


def _plane_wave_phases(ctx, idx):
    """k.r per grid point for the FFTW index triple idx, summed over the axes
    in the reference's order (src/solver.c:224-247): freq_d = 2 pi f_d / L_d
    with f_d the signed frequency, r_d = i_d L_d / N_d."""
    stride = [1, 1, 1]
    for d in range(1, ctx.dim):
        stride[d] = stride[d - 1] * ctx.N[d - 1]
    i = np.arange(ctx.size, dtype=np.int64)
    kr = np.zeros(ctx.size)
    for d in range(ctx.dim):
        f = idx[d] if idx[d] <= ctx.N[d] // 2 else idx[d] - ctx.N[d]
        freq = 2.0 * math.pi * float(f) / ctx.L[d]
        i_d = (i // stride[d]) % ctx.N[d]
        r_d = i_d.astype(np.float64) * ctx.L[d] / float(ctx.N[d])
        kr = kr + freq * r_d
    return kr


def planewave_block(ctx, m, hint=BDG_GEOM_AUTO):
    """BDG_INIT_PLANEWAVE block (src/solver.c:196-259 real, :381-412
    complex), as (m, n) rows: column j holds cos / sin (j even / odd) of
    wave vector (j + 1) // 2 of the |k|^2-sorted enumeration, plus a 1e-4
    xorshift32 perturbation (seed 42), times |psi0|, in both halves; columns
    past the enumerable wave vectors are xorshift32 noise (x - 1/2) |psi0|."""
    ent, n_k = enumerate_kvecs(ctx, hint, (m + 1) // 2)
    w = np.abs(ctx.wf) if ctx.wf is not None else np.ones(ctx.size)
    rng = XorShift32(42)
    S = ctx.size
    X = np.zeros((m, 2 * S), dtype=ctx.ctype)
    for j in range(m):
        kv = (j + 1) // 2
        draws = rng.xrand_many(S)
        if kv >= n_k:
            val = (draws - 0.5) * w
        else:
            kr = _plane_wave_phases(ctx, ent[kv][1])
            pw = np.sin(kr) if j % 2 == 1 else np.cos(kr)
            val = (pw + 1e-4 * (draws - 0.5)) * w
        X[j, :S] = val
        X[j, S:] = val
    return X


def wf_weighted_block_z(ctx, m):
    """Complex-path BDG_INIT_WF_WEIGHTED block (src/solver.c:331-345):
    |Box-Muller normal| |psi0| from the xorshift32 stream at seed 42 (two
    draws per entry, u1 clamped at 1e-10), in both halves, as (m, n) rows.
    (The real path seeds rand_r from time(NULL), src/solver.c:178-189, and
    has no reproducible block.)"""
    w = np.abs(ctx.wf) if ctx.wf is not None else np.ones(ctx.size)
    rng = XorShift32(42)
    S = ctx.size
    X = np.zeros((m, 2 * S), dtype=np.complex128)
    for j in range(m):
        d = rng.xrand_many(2 * S)
        u1 = np.fmax(d[0::2], 1e-10)
        u2 = d[1::2]
        val = np.abs(np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)) * w
        X[j, :S] = val
        X[j, S:] = val
    return X


def gaussian_block_bpositive(ctx, m, seed):
    """Seeded N(0,1) initial block made B-positive by setting v = u
    (the harness convention for configs that ask for X0 ~ N(0,1))."""
    rng = np.random.default_rng(seed)
    S = ctx.size
    if ctx.complex_psi0:
        u = rng.standard_normal((m, S)) + 1j * rng.standard_normal((m, S))
    else:
        u = rng.standard_normal((m, S))
    return np.concatenate([u, u], axis=1)


# ----------------------------------------------------------------------------
# iLOBPCG (restated from Kressner-Pandur-Shao 2014; block form)
# ----------------------------------------------------------------------------
def rr_pencil(Guu, Gvv, Guv, Ga, m, drop=1e-13, clamp=1e-14):
    """Rayleigh-Ritz for the projected definite pencil.

    Inputs are the Gram blocks of a basis S = [S_u; S_v] (k columns):
    Guu = S_u^H S_u, Gvv = S_v^H S_v, Guv = S_u^H S_v, Ga = S^H A S.
    Then S^H S = Guu + Gvv and S^H B S = Guv + Guv^H (B = swap).

    1. Standard-orthonormalise the basis implicitly (diagonal scaling + eigh
       of S^H S, directions below ``drop`` dropped): Z.
    2. On the orthonormal basis, factor A_s = Q D Q^H with D clamped at
       ``clamp * max(D)`` (keeps a near-null A direction such as the
       Goldstone mode finite) and form H = D^-1/2 Q^H B_s Q D^-1/2.
    3. Eigenpairs of H: theta = 1/lambda; positive-type eigenvalues are the
       positive theta; the m smallest positive lambda are the m largest theta.
    Returns lambda (ascending) and coefficients C (k x m) with
    C^H (S^H B S) C = I and C^H (S^H A S) C = diag(lambda)."""
    herm = lambda a: 0.5 * (a + a.conj().T)
    G = herm(Guu + Gvv)
    Gb = herm(Guv + Guv.conj().T)
    Ga = herm(Ga)
    dg = np.real(np.diag(G)).copy()
    dg[dg <= 0] = 1.0
    d = 1.0 / np.sqrt(dg)
    Gs = G * d[:, None] * d[None, :]
    s, Q = np.linalg.eigh(Gs)
    keep = s > drop * s.max()
    Z = (d[:, None] * Q[:, keep]) / np.sqrt(s[keep])[None, :]
    Ga2 = herm(Z.conj().T @ Ga @ Z)
    Gb2 = herm(Z.conj().T @ Gb @ Z)
    dA, Q2 = np.linalg.eigh(Ga2)
    dA = np.maximum(dA, clamp * dA.max())
    Y = Q2 / np.sqrt(dA)[None, :]
    H = herm(Y.conj().T @ Gb2 @ Y)
    th, Q3 = np.linalg.eigh(H)
    order = np.argsort(-th)
    npos = int(np.sum(th > 0))
    take = order[: min(m, npos)]
    C = Z @ Y @ Q3[:, take] / np.sqrt(th[take])[None, :]
    lam = 1.0 / th[take]
    return lam, C


class SolveResult:
    def __init__(self, lam, X, iters, nconv, true_res, history):
        self.eigvals = lam
        self.X = X
        self.iters = iters
        self.converged = nconv
        self.true_res = true_res
        self.history = history


def goldstone_projector(ctx, tol=1e-13, maxit=5000):
    """B-orthogonal projector onto the complement of the Goldstone Jordan
    chain {[psi0; 0], [0; w]} with M w = psi0.  Physical modes with
    omega != 0 satisfy psi0^H v = 0 and w^H u = 0.  w is computed by CG on M
    (Hermitian positive definite).  Holds for complex psi0 too, wherever
    K psi0 = 0; w^H psi0 = psi0^H M^-1 psi0 is real."""
    S = ctx.size
    psi = ctx.wf.astype(ctx.ctype)
    w = cg(lambda z: matmulM(ctx, z), psi, tol=tol, maxit=maxit)
    wpsi = np.vdot(w, psi)

    def proj(X):
        X = X.copy()
        u = X[:, :S]
        v = X[:, S:]
        a = (u @ np.conj(w)) / np.conj(wpsi)  # w^H u / w^H psi
        b = (v @ np.conj(psi)) / wpsi  # psi^H v / psi^H w
        X[:, :S] = u - a[:, None] * psi[None, :]
        X[:, S:] = v - b[:, None] * w[None, :]
        return X

    return proj, w


def cg(apply, b, tol=1e-13, maxit=5000, x0=None):
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - apply(x) if x0 is not None else b.copy()
    p = r.copy()
    rr = np.vdot(r, r).real
    bn = math.sqrt(np.vdot(b, b).real)
    for _ in range(maxit):
        if math.sqrt(rr) <= tol * bn:
            break
        Ap = apply(p)
        alpha = rr / np.vdot(p, Ap).real
        x = x + alpha * p
        r = r - alpha * Ap
        rr_new = np.vdot(r, r).real
        p = r + (rr_new / rr) * p
        rr = rr_new
    return x


def true_residual(ctx, X, AX, lam, ncols):
    """||K M v - lambda^2 v|| / ||v|| per column; M v is the lower half of AX."""
    S = ctx.size
    Mv = AX[:ncols, S:]
    KMv = matmulK(ctx, Mv)
    v = X[:ncols, S:]
    r = KMv - (lam[:ncols] ** 2)[:, None] * v
    return np.linalg.norm(r, axis=1) / np.maximum(np.linalg.norm(v, axis=1), 1e-300)


def gram_blocks(ctx, S_, AS_):
    S = ctx.size
    Su, Sv = S_[:, :S], S_[:, S:]
    Guu = Su.conj() @ Su.T
    Gvv = Sv.conj() @ Sv.T
    Guv = Su.conj() @ Sv.T
    Ga = S_.conj() @ AS_.T
    return Guu, Gvv, Guv, Ga


def anorm_estimate(ctx):
    """Upper bound of ||A|| = max(||K||, ||M||) used to scale the backward-error
    convergence test: max kinetic energy of the grid plus the largest local
    term (plus the dipolar exchange bound when active)."""
    kin = 0.5 * sum(float(np.max(k)) for k in ctx.kx2)
    aK = float(np.max(np.abs(ctx.localTermK)))
    aM = float(np.max(np.abs(ctx.localTermM)))
    if ctx.dipolar and ctx.dim == 3:
        aM += 2.0 * abs(ctx.g_ddi) * float(np.max(np.abs(ctx.wf)) ** 2) * \
            float(np.max(np.abs(ctx.longRngInt)))
    return kin + max(aK, aM)


CONV_BACKWARD, CONV_TRUE_RESIDUAL = 0, 1


def residual_measure(ctx, X, AX, lam, ncols, criterion, anorm):
    """Per-column convergence measure.

    CONV_BACKWARD: ||A x - lam B x|| / ((||A||_est + |lam|) ||x||)
    CONV_TRUE_RESIDUAL: ||K M v - lam^2 v|| / ||v|| (the BdG residual)."""
    if criterion == CONV_TRUE_RESIDUAL:
        return true_residual(ctx, X, AX, lam, ncols)
    S = ctx.size
    Xs, AXs, l = X[:ncols], AX[:ncols], lam[:ncols]
    R = AXs - l[:, None] * np.concatenate([Xs[:, S:], Xs[:, :S]], axis=1)
    return np.linalg.norm(R, axis=1) / ((anorm + np.abs(l)) * np.linalg.norm(Xs, axis=1))


def _scaled_eigh(G, drop):
    """eigh of D G D with D = diag(G)^-1/2; returns d, s, Q, keep-mask of
    the directions above ``drop * max(s)``."""
    dg = np.real(np.diag(G)).copy()
    dg[dg <= 0] = 1.0
    d = 1.0 / np.sqrt(dg)
    s, Q = np.linalg.eigh(0.5 * (G + G.conj().T) * d[:, None] * d[None, :])
    keep = s > drop * s.max()
    return d, s, Q, keep


def gram_pinv(G, drop=1e-13):
    """Pseudo-inverse of a Gram matrix, dropping near-dependent directions."""
    d, s, Q, keep = _scaled_eigh(G, drop)
    Qk = Q[:, keep]
    return (d[:, None] * Qk / s[keep][None, :]) @ (Qk.conj().T * d[None, :])


def svqb_coeffs(G, drop=1e-13):
    """Z with Z^H G Z = I on the kept directions (SVQB, Stathopoulos & Wu
    2002): V Z is an orthonormal basis of span V, dependent directions
    dropped."""
    d, s, Q, keep = _scaled_eigh(G, drop)
    return d[:, None] * Q[:, keep] / np.sqrt(s[keep])[None, :]


def ilobpcg(ctx, X0, nev, maxIter, tol, proj=None, applyA=None, applyT=None,
            criterion=CONV_BACKWARD, lock=True, drop=1e-13, guard=1e-4, guard_strict=1e-12, stall_win=10,
            project_p=True, normalize_p=False, verbose=False):
    """Block iLOBPCG for the pencil (A, B) = (diag(K, M), swap).

    X0: (m, n) block (rows are the columns of the reference's S), B-positive.
    Per iteration (the GPU solver runs the same steps):
      R = A X - B X diag(lam) on the active columns, W = T R
      (project_p only: P <- P - X (X^H X)^+ X^H P, AP alike; SVQB-normalised
      as well only with normalize_p)
      W <- W - Q (Q^H Q)^+ Q^H W with Q = [X, P], then SVQB-normalised
      Rayleigh-Ritz on S = [X, P, W]  (rr_pencil)
      X <- S C,  P <- [P, W] C_pw  (restricted to the active columns)
    Active columns: wanted (j < nev) while their measure exceeds tol,
    guards (j >= nev) while their backward error exceeds the guard level:
    `guard` (1e-4) while the worst backward error of the unconverged wanted
    pairs keeps halving within every `stall_win` iterations, `guard_strict`
    (1e-12) for the rest of the solve once it does not (loose guards can hold
    the wanted pairs above tol, e.g. with an undeflated zero mode wanted).
    Converged when the measure is <= tol for each of the first nev pairs.

    P is re-projected against X and SVQB-normalised each iteration
    (project_p).  Without it the small cases converge alike (16^3 42 / 42,
    32^3 78 / 78 iterations), but on the GPU the 128^3 FP64 solve stalled at a
    true residual of 1.2e-8 for 4 of 32 pairs, so the projection stays.  Its
    SVQB normalisation does not: the W projection's pseudo-inverse and the
    Rayleigh-Ritz step's scaled eigen-decomposition drop the dependent
    directions of the projected P (32^3 78 / 78, 64^3 65 / 66 iterations with
    and without it, eigenvalues to 5e-15; 128^3 on the GPU 63 / 63)."""
    A = applyA or (lambda Z: matmulLrep(ctx, Z))
    T = applyT or (lambda Z: precondLrep(ctx, Z))
    anorm = anorm_estimate(ctx)
    m = X0.shape[0]
    X = proj(X0) if proj else X0.copy()
    AX = A(X)
    lam, C = rr_pencil(*gram_blocks(ctx, X, AX), m, drop=drop)
    if len(lam) < m:
        raise RuntimeError("initial block is not B-positive")
    X = C.T @ X
    AX = C.T @ AX
    P = AP = None
    history = []
    it = 0
    res = None
    nconv = 0
    guard_now = guard
    worst_hist = []
    while True:
        back = residual_measure(ctx, X, AX, lam, m, CONV_BACKWARD, anorm)
        res = back[:nev] if criterion == CONV_BACKWARD else \
            residual_measure(ctx, X, AX, lam, nev, criterion, anorm)
        nconv = int(np.sum(res <= tol))
        unconv = res > tol
        worst = float(np.max(back[:nev][unconv])) if np.any(unconv) else 0.0
        worst_hist.append(worst)
        if guard_now != guard_strict and len(worst_hist) > stall_win and \
                not worst <= 0.5 * worst_hist[-1 - stall_win]:
            guard_now = guard_strict
        history.append((lam[:nev].copy(), res.copy()))
        if verbose:
            print(it, lam[:nev], res.max())
        if nconv >= nev or it >= maxIter:
            break
        if lock:
            act = np.concatenate([np.where(res > tol)[0], nev + np.where(back[nev:] > guard_now)[0]])
        else:
            act = np.arange(m)
        R = AX[act] - lam[act, None] * matmulSwap(ctx, X[act])
        W = T(R)
        if proj:
            W = proj(W)
        if project_p and P is not None and len(P):
            Cpx = gram_pinv(X.conj() @ X.T, drop) @ (X.conj() @ P.T)
            P = P - Cpx.T @ X
            AP = AP - Cpx.T @ AX
            if normalize_p:
                Z = svqb_coeffs(P.conj() @ P.T, drop)
                P = Z.T @ P
                AP = Z.T @ AP
        Q = X if P is None else np.concatenate([X, P])
        Y = gram_pinv(Q.conj() @ Q.T, drop) @ (Q.conj() @ W.T)
        W = W - Y.T @ Q
        W = svqb_coeffs(W.conj() @ W.T, drop).T @ W
        AW = A(W)
        S_ = np.concatenate([Q, W])
        AS_ = np.concatenate([AX, AW] if P is None else [AX, AP, AW])
        lam_new, C = rr_pencil(*gram_blocks(ctx, S_, AS_), m, drop=drop)
        if len(lam_new) < m:
            raise RuntimeError("lost B-positivity of the search space")
        Cr = C[m:]
        Pn = Cr.T @ S_[m:]
        APn = Cr.T @ AS_[m:]
        X = C[:m].T @ X + Pn
        AX = C[:m].T @ AX + APn
        P, AP = Pn[act], APn[act]
        lam = lam_new
        it += 1
    return SolveResult(lam, X, it, nconv, res, history)


# ----------------------------------------------------------------------------
# ground state by split-step imaginary-time propagation (harness input)
# ----------------------------------------------------------------------------
def itp_ground_state(N, L, omegas, g, gdd=0.0, dipole_dir=(0.0, 0.0, 1.0),
                     Rc=None, dt=1e-3, tol=1e-12, max_steps=200000,
                     vortex=False, verbose=False):
    """Split-step (Strang) imaginary-time propagation from a unit Gaussian
    (times (x+iy)/r with the phase held fixed when ``vortex``).

    H = -1/2 lap + V + g|psi|^2 + gdd * F^-1[Vdd F|psi|^2], normalised to
    sum |psi|^2 dV = 1 on the grid x_i = (i - N/2) L/N.  Stops when the
    per-step change of mu = <psi|H|psi> is below ``tol``.
    Returns (psi, mu, steps)."""
    dim = len(N)
    ctx = Ctx(dim, N, L, complex_psi0=vortex)
    set_system(ctx)
    dV = float(np.prod([l / n for l, n in zip(L, N)]))
    V = harmonic_trap(ctx, omegas).reshape(ctx.rshape)
    c = grid_coords(ctx)
    mesh = list(reversed(np.meshgrid(*reversed(c), indexing="ij")))
    r2 = sum(m * m for m in mesh)
    psi = np.exp(-0.5 * r2).astype(np.complex128 if vortex else np.float64)
    phase = None
    if vortex:
        phase = np.exp(1j * np.arctan2(mesh[1], mesh[0]))
        rr = np.sqrt(mesh[0] ** 2 + mesh[1] ** 2)
        psi = psi * rr * phase
    psi /= math.sqrt(np.sum(np.abs(psi) ** 2) * dV)
    k2 = ctx.k2.reshape(ctx.kshape)
    half_kin = np.exp(-0.25 * dt * k2)
    if gdd != 0.0:
        dipolar_set_kernel(ctx, gdd, dipole_dir, Rc)
        vdd = ctx.longRngInt.reshape(ctx.kshape) / ctx.size
    else:
        vdd = None
    fw = (lambda a: sfft.fftn(a, workers=_WORKERS)) if vortex else (lambda a: sfft.rfftn(a, workers=_WORKERS))
    bw = ((lambda A: sfft.ifftn(A, workers=_WORKERS)) if vortex
          else (lambda A: sfft.irfftn(A, s=ctx.rshape, workers=_WORKERS)))

    def potential(p):
        n = np.abs(p) ** 2
        U = V + g * n
        if vdd is not None:
            if vortex:  # the kernel is on the full spectrum of the complex context
                phi = np.real(sfft.ifftn(sfft.fftn(n, workers=_WORKERS) * vdd, norm="forward",
                                         workers=_WORKERS))
            else:
                phi = sfft.irfftn(sfft.rfftn(n, workers=_WORKERS) * vdd, s=ctx.rshape,
                                  norm="forward", workers=_WORKERS)
            U = U + gdd * phi
        return U

    def mu_of(p):
        kin = bw(0.5 * k2 * fw(p))
        Hp = kin + potential(p) * p
        return float(np.real(np.sum(np.conj(p) * Hp)) / np.sum(np.abs(p) ** 2))

    mu_old = mu_of(psi)
    steps = 0
    for steps in range(1, max_steps + 1):
        psi = bw(half_kin * fw(psi))
        psi = psi * np.exp(-dt * potential(psi))
        psi = bw(half_kin * fw(psi))
        if vortex:
            psi = np.abs(psi) * phase
        psi /= math.sqrt(np.sum(np.abs(psi) ** 2) * dV)
        mu = mu_of(psi)
        if verbose and steps % 1000 == 0:
            print(steps, mu, mu - mu_old)
        if abs(mu - mu_old) < tol:
            mu_old = mu
            break
        mu_old = mu
    return psi.reshape(-1), mu_old, steps


def newton_polish(N, L, omegas, g, gdd, psi, Rc=None, dipole_dir=(0.0, 0.0, 1.0), tol=1e-13, maxit=8):
    """Polish a real ground state to the exact stationary state of the
    discrete GPE (split-step ITP stops at an O(dt^2) splitting error, which
    leaves K psi0 != 0).  Bordered Newton on F(psi, mu) = H(psi) psi - mu psi
    with the normalisation constraint: the Jacobian of F is the BdG operator
    M, so each step solves M a = r and M b = psi by CG and sets
    delta = -a + dmu b with psi^T delta = 0.  Returns (psi, mu, |r|)."""
    dV = float(np.prod([l / n for l, n in zip(L, N)]))
    psi = np.asarray(psi, dtype=np.float64).copy()
    rn = float("inf")
    mu = 0.0
    for _ in range(maxit + 1):
        c = build_problem(N, L, omegas, g, gdd, psi, 0.0, dipole_dir, Rc)
        Hp = matmulK(c, psi)
        mu = float(np.dot(psi, Hp) / np.dot(psi, psi))
        r = Hp - mu * psi
        rn = float(np.linalg.norm(r) * math.sqrt(dV))
        if rn < tol:
            break
        c = build_problem(N, L, omegas, g, gdd, psi, mu, dipole_dir, Rc)
        Mop = lambda z: matmulM(c, z)
        a = cg(Mop, r, tol=1e-14, maxit=10000)
        b = cg(Mop, psi, tol=1e-14, maxit=10000)
        dmu = float(np.dot(psi, a) / np.dot(psi, b))
        psi = psi - a + dmu * b
        psi /= math.sqrt(np.sum(psi * psi) * dV)
    return psi, mu, rn


def build_problem(N, L, omegas, g, gdd, psi, mu, dipole_dir=(0.0, 0.0, 1.0),
                  Rc=None, complex_psi0=False):
    """Assemble the BdG context the way the reference's setup chain does
    (set_system, trap, wavefunction, contact interactions U_K = U_M = g n,
    dipolar, mu)."""
    ctx = Ctx(len(N), N, L, complex_psi0)
    set_system(ctx)
    set_trap_array(ctx, harmonic_trap(ctx, omegas))
    set_wavefunction(ctx, psi)
    set_local_interactions(ctx, lambda n: g * n, lambda n: g * n)
    if gdd != 0.0:
        set_dipolar(ctx, gdd, dipole_dir, Rc)
    set_mu(ctx, mu)
    return ctx
