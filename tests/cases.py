"""Known-answer operator cases of the reference's own unit tests.

Each case restates one assertion block of pstuermer/BDG_LOBPCG tests/test_*.c
(file:line in the docstring) as (setup, input, expected output, tolerance)
and runs against an *adapter*: the CPU oracle (tests/test_oracle_cpu.py) or
the GPU library (test_known_answer_gpu in tests/test_ops_gpu.py).  Same inputs, same
tolerances as the reference (1e-10 absolute unless stated).
"""
import math

import numpy as np

TWO_PI = 2.0 * math.pi


class OracleAdapter:
    def __init__(self, dim, N, L, cplx=False):
        from oracle import bdg_oracle as O

        self.O = O
        self.c = O.Ctx(dim, N, L, cplx)
        O.set_system(self.c)
        self.cplx = cplx

    def set(self, name, arr):
        dt = np.complex128 if (name == "wf" and self.cplx) else np.float64
        setattr(self.c, name, np.asarray(arr, dtype=dt).reshape(-1).copy())

    def set_scalar(self, name, v):
        setattr(self.c, name, v)

    def set_dipolar_kernel(self, g, d, rc):
        self.O.dipolar_set_kernel(self.c, g, d, rc)

    def kernel(self):
        return self.c.longRngInt

    def add_meanfield(self):
        self.O.dipolar_add_meanfield(self.c)

    def get(self, name):
        return getattr(self.c, name)

    def apply(self, op, x):
        return getattr(self.O, op)(self.c, np.asarray(x))


class GpuAdapter:
    def __init__(self, dim, N, L, cplx=False):
        import bdg_lobpcg_b200 as B

        self.c = B.OperatorContext(dim, N, L, cplx)
        self.cplx = cplx

    def set(self, name, arr):
        self.c.set(name, arr)

    def set_scalar(self, name, v):
        self.c.set_scalar(name, v)

    def set_dipolar_kernel(self, g, d, rc):
        self.c.set_dipolar_kernel(g, d, rc)

    def kernel(self):
        return self.c.get("longRngInt").copy()

    def add_meanfield(self):
        self.c.add_meanfield()

    def get(self, name):
        return self.c.get(name).copy()

    def apply(self, op, x):
        return self.c.apply(op, x)


def grid1(N, L=TWO_PI):
    return np.arange(N) * L / N


def grid3(N, L=(TWO_PI,) * 3):
    x = np.arange(N[0]) * L[0] / N[0]
    y = np.arange(N[1]) * L[1] / N[1]
    z = np.arange(N[2]) * L[2] / N[2]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X.reshape(-1), Y.reshape(-1), Z.reshape(-1)


def _lt(ad, size, K, M):
    ad.set("localTermK", np.full(size, K))
    ad.set("localTermM", np.full(size, M))


def _pre(ad, size, V0K, V0M, mu):
    ad.set("localTermK", np.full(size, V0K - mu))
    ad.set("localTermM", np.full(size, V0M - mu))
    ad.set("precond_sqrtK", np.full(size, 1.0 / math.sqrt(V0K)))
    ad.set("precond_sqrtM", np.full(size, 1.0 / math.sqrt(V0M)))
    ad.set_scalar("mu", mu)


# --------------------------------------------------------------------------
# each case: f(make_adapter) -> list of (got, expected, tol) triples
# --------------------------------------------------------------------------
def kinetic_planewave_1d(make):
    """tests/test_kinetic.c:45-71: cos x -> 0.5 cos x (N=64, L=2pi)."""
    ad = make(1, [64], [TWO_PI])
    x = grid1(64)
    return [(ad.apply("kinetic", np.cos(x)), 0.5 * np.cos(x), 1e-10)]


def kinetic_superposition_1d(make):
    """tests/test_kinetic.c:77-104: cos x + 0.5 cos 3x -> 0.5 cos x + 2.25 cos 3x."""
    ad = make(1, [64], [TWO_PI])
    x = grid1(64)
    return [(ad.apply("kinetic", np.cos(x) + 0.5 * np.cos(3 * x)), 0.5 * np.cos(x) + 2.25 * np.cos(3 * x), 1e-10)]


def kinetic_z_matches_d(make):
    """tests/test_kinetic.c:109-143: complex path on a real input equals the real path."""
    x = np.cos(grid1(64))
    yd = make(1, [64], [TWO_PI]).apply("kinetic", x)
    yz = make(1, [64], [TWO_PI], True).apply("kinetic", x.astype(np.complex128))
    return [(yz.real, yd, 1e-10), (yz.imag, 0 * yd, 1e-10)]


def kinetic_planewave_3d(make):
    """tests/test_kinetic.c:148-180: cos(x+y+z) on 16^3 -> 1.5 cos(x+y+z)."""
    ad = make(3, [16] * 3, [TWO_PI] * 3)
    X, Y, Z = grid3([16] * 3)
    f = np.cos(X + Y + Z)
    return [(ad.apply("kinetic", f), 1.5 * f, 1e-10)]


def kinetic_zero_mode(make):
    """tests/test_kinetic.c:185-205: constant -> 0 (N=32)."""
    ad = make(1, [32], [TWO_PI])
    return [(ad.apply("kinetic", np.ones(32)), np.zeros(32), 1e-10)]


def matmulK_planewave_1d(make):
    """tests/test_matmulK.c:69-94: K cos x with V0=2, mu=0 -> 2.5 cos x."""
    ad = make(1, [64], [TWO_PI])
    _lt(ad, 64, 2.0, 2.0)
    x = grid1(64)
    return [(ad.apply("matmulK", np.cos(x)), 2.5 * np.cos(x), 1e-10)]


def matmulK_constant(make):
    """tests/test_matmulK.c:100-120: K 1 with V0=3, mu=1 -> 2."""
    ad = make(1, [32], [TWO_PI])
    _lt(ad, 32, 2.0, 2.0)
    return [(ad.apply("matmulK", np.ones(32)), np.full(32, 2.0), 1e-10)]


def matmulK_dz(make):
    """tests/test_matmulK.c:125-165: d and z paths agree (V0=2, mu=0.5)."""
    x = np.cos(grid1(64)) + 0.3 * np.sin(2 * grid1(64))
    ad = make(1, [64], [TWO_PI])
    _lt(ad, 64, 1.5, 1.5)
    az = make(1, [64], [TWO_PI], True)
    _lt(az, 64, 1.5, 1.5)
    yd = ad.apply("matmulK", x)
    yz = az.apply("matmulK", x.astype(np.complex128))
    return [(yz.real, yd, 1e-10), (yz.imag, 0 * yd, 1e-10)]


def matmulK_3d(make):
    """tests/test_matmulK.c:172-215: 16^3 cos(x+y+z), V=1 -> 2.5 cos."""
    ad = make(3, [16] * 3, [TWO_PI] * 3)
    _lt(ad, 16 ** 3, 1.0, 1.0)
    X, Y, Z = grid3([16] * 3)
    f = np.cos(X + Y + Z)
    return [(ad.apply("matmulK", f), 2.5 * f, 1e-10)]


def matmulM_no_dipolar(make):
    """tests/test_matmulM.c:67-88: M cos x with VM=2 -> 2.5 cos x."""
    ad = make(1, [64], [TWO_PI])
    _lt(ad, 64, 0.0, 2.0)
    x = grid1(64)
    return [(ad.apply("matmulM", np.cos(x)), 2.5 * np.cos(x), 1e-10)]


def matmulM_matches_K(make):
    """tests/test_matmulM.c:93-121: equal local terms, no dipolar -> M == K."""
    x = grid1(64)
    f = np.cos(x) + 0.5 * np.cos(3 * x)
    ad = make(1, [64], [TWO_PI])
    _lt(ad, 64, 1.5, 1.5)
    return [(ad.apply("matmulM", f), ad.apply("matmulK", f), 1e-10)]


def matmulM_dz(make):
    """tests/test_matmulM.c:126-162: d/z consistency without dipolar."""
    f = np.cos(grid1(64))
    ad = make(1, [64], [TWO_PI])
    _lt(ad, 64, 0.0, 2.0)
    az = make(1, [64], [TWO_PI], True)
    _lt(az, 64, 0.0, 2.0)
    yd = ad.apply("matmulM", f)
    yz = az.apply("matmulM", f.astype(np.complex128))
    return [(yz.real, yd, 1e-10), (yz.imag, 0 * yd, 1e-10)]


def _dip3(make, cplx, wfval, ltK, ltM, g=1.0):
    N = [8, 8, 8]
    ad = make(3, N, [TWO_PI] * 3, cplx)
    _lt(ad, 512, ltK, ltM)
    ad.set("wf", wfval)
    ad.set_dipolar_kernel(g, [0.0, 0.0, 1.0], TWO_PI / 2.0)
    ad.set_scalar("dipolar", 1)
    return ad


def matmulM_3d_dipolar_nonzero(make):
    """tests/test_matmulM.c:171-222: dipolar term present for cos z (max |M-K| > 1e-6)."""
    ad = _dip3(make, False, np.ones(512), 1.0, 1.0)
    X, Y, Z = grid3([8] * 3)
    f = np.cos(Z)
    d = np.max(np.abs(ad.apply("matmulM", f) - ad.apply("matmulK", f)))
    return [(np.array([float(d > 1e-6)]), np.array([1.0]), 0.5)]


def matmulM_3d_dipolar_dz(make):
    """tests/test_matmulM.c:227-282: 3D dipolar M, d vs z."""
    i = np.arange(512)
    w = 1.0 + 0.1 * (i % 7)
    ad = _dip3(make, False, w, 1.0, 1.5)
    az = _dip3(make, True, w.astype(np.complex128), 1.0, 1.5)
    f = np.sin(TWO_PI * (i % 8) / 8)
    yd = ad.apply("matmulM", f)
    yz = az.apply("matmulM", f.astype(np.complex128))
    return [(yz.real, yd, 1e-10), (yz.imag, 0 * yd, 1e-10)]


def precond_planewave(make, which="precondK", cplx=False):
    N, mu = 64, 0.5
    ad = make(1, [N], [TWO_PI], cplx)
    VK, VM = 2.0, 3.5
    _pre(ad, N, VK, VM, mu)
    x = grid1(N)
    V0 = VK if which == "precondK" else VM
    y = ad.apply(which, np.cos(x).astype(np.complex128 if cplx else np.float64))
    exp = np.cos(x) / (V0 * (mu + 0.5))
    out = [(y.real, exp, 1e-10)]
    if cplx:
        out.append((y.imag, 0 * exp, 1e-10))
    return out


def precondK_d_planewave(make):
    """tests/test_precond.c:71-101: T_K cos x = cos x / (V0 (mu + 1/2))."""
    return precond_planewave(make, "precondK", False)


def precondK_z_planewave(make):
    """tests/test_precond.c:103-131 (complex path)."""
    return precond_planewave(make, "precondK", True)


def precondM_d_planewave(make):
    """tests/test_precond.c:170-215: T_M with VM = 3.5."""
    return precond_planewave(make, "precondM", False)


def precond_zero_mode(make):
    """tests/test_precond.c:~370-392: T_K 1 = 1/(V0 mu) (V0=2, mu=1.5)."""
    ad = make(1, [64], [TWO_PI])
    _pre(ad, 64, 2.0, 2.0, 1.5)
    return [(ad.apply("precondK", np.ones(64)), np.full(64, 1.0 / (2.0 * 1.5)), 1e-10)]


def precond_dz(make):
    """tests/test_precond.c:133-165: T_K d vs z (V0=3, mu=1)."""
    x = grid1(64)
    f = np.cos(x) + 0.3 * np.sin(2 * x)
    ad = make(1, [64], [TWO_PI])
    _pre(ad, 64, 3.0, 3.0, 1.0)
    az = make(1, [64], [TWO_PI], True)
    _pre(az, 64, 3.0, 3.0, 1.0)
    yd = ad.apply("precondK", f)
    yz = az.apply("precondK", f.astype(np.complex128))
    return [(yz.real, yd, 1e-10), (yz.imag, 0 * yd, 1e-10)]


def precondLrep_block(make):
    """tests/test_precond.c:220-270: T_Lrep = [T_K u; T_M v]."""
    ad = make(1, [64], [TWO_PI])
    _pre(ad, 64, 2.0, 3.5, 0.5)
    x = grid1(64)
    u = np.cos(x)
    v = np.sin(2 * x) + 0.2
    y = ad.apply("precondLrep", np.concatenate([u, v]))
    return [(y[:64], ad.apply("precondK", u), 1e-10), (y[64:], ad.apply("precondM", v), 1e-10)]


def lrep_block(make):
    """tests/test_matmulLrep.c:68-148: Lrep = [K u; M v]."""
    ad = make(1, [64], [TWO_PI])
    _lt(ad, 64, 1.0, 2.5)
    x = grid1(64)
    u = np.cos(x)
    v = np.cos(2 * x) + 0.1
    y = ad.apply("matmulLrep", np.concatenate([u, v]))
    return [(y[:64], ad.apply("matmulK", u), 1e-15 + 1e-13), (y[64:], ad.apply("matmulM", v), 1e-13)]


def swap_block(make):
    """tests/test_matmulSwap.c:52-100: swap halves and involution (TOL 1e-15)."""
    ad = make(1, [8], [TWO_PI])
    x = np.arange(16) * 0.7 + 0.7
    y = ad.apply("matmulSwap", x)
    return [(y, np.concatenate([x[8:], x[:8]]), 1e-15), (ad.apply("matmulSwap", y), x, 1e-15)]


def dipolar_kernel_values(make):
    """tests/test_dipolar.c:44-109: kernel(0)=0, kernel(k_z)=2C(pi), kernel(k_x)=-C(pi)."""
    ad = make(3, [8] * 3, [TWO_PI] * 3)
    ad.set_dipolar_kernel(1.0, [0.0, 0.0, 1.0], math.pi)
    k = ad.kernel()
    kR = math.pi
    fc = 1.0 + 3.0 * math.cos(kR) / kR ** 2 - 3.0 * math.sin(kR) / kR ** 3
    return [(np.array([k[0], k[1 * 8 * 5], k[1]]), np.array([0.0, 2.0 * fc, -fc]), 1e-10)]


def dipolar_kernel_r2c_vs_c2c(make):
    """tests/test_dipolar.c:117-150: r2c and c2c kernels agree on shared points."""
    ar = make(3, [8] * 3, [TWO_PI] * 3)
    ac = make(3, [8] * 3, [TWO_PI] * 3, True)
    ar.set_dipolar_kernel(1.0, [0, 0, 1.0], math.pi)
    ac.set_dipolar_kernel(1.0, [0, 0, 1.0], math.pi)
    kr = ar.kernel().reshape(8, 8, 5)
    kc = ac.kernel().reshape(8, 8, 8)
    return [(kr, kc[:, :, :5], 1e-10)]


def meanfield_uniform(make):
    """tests/test_dipolar.c:156-181: uniform density -> zero mean field (1e-12)."""
    ad = make(3, [8] * 3, [TWO_PI] * 3)
    _lt(ad, 512, 0.0, 0.0)
    ad.set("wf", np.ones(512))
    ad.set_dipolar_kernel(1.0, [0, 0, 1.0], math.pi)
    ad.add_meanfield()
    return [(ad.get("localTermK"), np.zeros(512), 1e-12), (ad.get("localTermM"), np.zeros(512), 1e-12)]


def meanfield_dz(make):
    """tests/test_dipolar.c:187-231: mean field d vs z for wf = 1 + 0.3 cos(x+y+z)."""
    X, Y, Z = grid3([8] * 3)
    w = 1.0 + 0.3 * np.cos(X + Y + Z)
    out = []
    res = []
    for cplx in (False, True):
        ad = make(3, [8] * 3, [TWO_PI] * 3, cplx)
        _lt(ad, 512, 0.0, 0.0)
        ad.set("wf", w.astype(np.complex128) if cplx else w)
        ad.set_dipolar_kernel(1.0, [0, 0, 1.0], math.pi)
        ad.add_meanfield()
        res.append((ad.get("localTermK"), ad.get("localTermM")))
    out.append((res[1][0], res[0][0], 1e-10))
    out.append((res[1][1], res[0][1], 1e-10))
    return out


def dipolar_conv_linearity(make):
    """tests/test_dipolar.c:236-266: conv(3.7 v) = 3.7 conv(v) (g=1.5)."""
    ad = make(3, [8] * 3, [TWO_PI] * 3)
    i = np.arange(512)
    ad.set("wf", 1.0 + 0.1 * (i % 7))
    ad.set_dipolar_kernel(1.5, [0, 0, 1.0], math.pi)
    v = np.cos(TWO_PI * (i % 8) / 8)
    return [(ad.apply("dipolar_conv", 3.7 * v), 3.7 * ad.apply("dipolar_conv", v), 1e-10)]


def dipolar_conv_dz(make):
    """tests/test_dipolar.c:271-309: dipolar conv d vs z."""
    i = np.arange(512)
    w = 1.0 + 0.2 * (i % 5)
    v = np.sin(TWO_PI * (i % 8) / 8)
    ad = make(3, [8] * 3, [TWO_PI] * 3)
    ad.set("wf", w)
    ad.set_dipolar_kernel(1.0, [0, 0, 1.0], math.pi)
    az = make(3, [8] * 3, [TWO_PI] * 3, True)
    az.set("wf", w.astype(np.complex128))
    az.set_dipolar_kernel(1.0, [0, 0, 1.0], math.pi)
    yd = ad.apply("dipolar_conv", v)
    yz = az.apply("dipolar_conv", v.astype(np.complex128))
    return [(yz.real, yd, 1e-10), (yz.imag, 0 * yd, 1e-10)]


def k_tables(make):
    """tests/test_setup.c:49-190: k_size, kx2 and k2 values (L = 2pi)."""
    ad = make(3, [8, 8, 8], [TWO_PI] * 3)
    k2 = ad.get("k2").reshape(8, 8, 5)
    n0 = 5
    return [(np.array([k2[1, 0, 0], k2[1, 1, 1], k2[5, 3, 2], k2.size]), np.array([1.0, 3.0, 22.0, 8 * 8 * n0]), 1e-12)]


CASES = [kinetic_planewave_1d, kinetic_superposition_1d, kinetic_z_matches_d, kinetic_planewave_3d,
         kinetic_zero_mode, matmulK_planewave_1d, matmulK_constant, matmulK_dz, matmulK_3d,
         matmulM_no_dipolar, matmulM_matches_K, matmulM_dz, matmulM_3d_dipolar_nonzero,
         matmulM_3d_dipolar_dz, precondK_d_planewave, precondK_z_planewave, precondM_d_planewave,
         precond_zero_mode, precond_dz, precondLrep_block, lrep_block, swap_block, dipolar_kernel_values,
         dipolar_kernel_r2c_vs_c2c, meanfield_uniform, meanfield_dz, dipolar_conv_linearity, dipolar_conv_dz,
         k_tables]


def check(triples):
    for got, exp, tol in triples:
        got = np.asarray(got)
        exp = np.asarray(exp)
        assert got.shape == exp.shape, (got.shape, exp.shape)
        err = float(np.max(np.abs(got - exp))) if got.size else 0.0
        assert err < tol, f"max abs error {err:.3e} >= {tol:.1e}"
