"""CPU restatement (numpy, FP64) of the learned SPD preconditioner.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA forward, adjoint, gradient
and Adam kernels of bdg_lobpcg_b200/csrc/bdg_learn.cu.  The product path
never imports it.  The reference has no learned preconditioner (its
preconditioner is the diagonal k-space one of src/precond_impl.inc:21-118,
restated in oracle/bdg_oracle.py); this component has no counterpart there,
so its parity is pinned by finite differences of its own loss (gradient) and
by the exact algebraic properties the construction guarantees (symmetry and
positivity of T).

The preconditioner for one half (K or M) of the BdG block is

    T r = S^T S r + exp(eta) P0 r,

P0 the plain k-space preconditioner of that half and S a linear map of r
onto C channels on the 2x coarsened grid (n = N/2 per axis):

    rc    = D r                    2x2x2 average pooling
    z0[c] = a_c * rc               lift, a_c = sum_f A[c, f] phi_f
    z_l   = z_{l-1} + SC_l(z_{l-1}) + PM_l(z_{l-1}),   l = 1..L
    S r   = z_L

phi_f are conditioning fields on the coarse grid: 1, the condensate density
|psi0|^2 / max, the trap V / max|V|, eps_dd and lambda / 4 (constants).
SC_l is a spectral convolution over the lowest `modes` wave numbers per axis
with a filter even in each wave-number component, written in a real basis:
per axis the rows cos(2 pi a x / n), a = 0..modes-1, and sin(2 pi a x / n),
a = 1..modes-1 (R = 2 modes - 1 rows), P = E_z (x) E_y (x) E_x, and

    SC_l(z)[c] = P^T (w_l[c] * (P z[c])),
    w_l[c][i, j, k] = W_l[c][a_i, a_j, a_k] m_i m_j m_k / n^3

(m = 1 for a = 0, else 2), which equals F^-1 (G F z) / n^3 for the even
filter G; P^T diag(w) P is symmetric, so SC_l is self-adjoint.  PM_l is a
pointwise channel mix with a conditioned diagonal:

    PM_l(z)[c] = sum_c' B_l[c, c'] z[c'] + (sum_f Dg_l[c, f] phi_f) z[c].

S^T applies the adjoints in reverse order; T is symmetric positive definite
whenever P0 is.  Training minimises, over pairs (r, e), either ||T r - e||^2 / ||e||^2
(with d = T r - e the gradient is 2 / ||e||^2 grad_theta <S d, S r>, d and
r held fixed, and 2 exp(eta) <d, P0 r> / ||e||^2 for eta) or the energy
norm ||T r - e||_A^2 / ||e||_A^2 with e = A^-1 r (loss_and_grad_energy:
the same form with d = A T r - r and <r, e> in place of ||e||^2).
"""
import numpy as np

C_DEF, L_DEF, MODES_DEF, NFEAT = 16, 4, 12, 5


def basis(n, modes):
    """Per-axis rows (R x n): cos rows a = 0..modes-1, sin rows a = 1..modes-1,
    their wave number a and multiplicity m."""
    x = np.arange(n)
    rows, a, m = [], [], []
    for k in range(modes):
        rows.append(np.cos(2 * np.pi * k * x / n))
        a.append(k)
        m.append(1.0 if k == 0 else 2.0)
    for k in range(1, modes):
        rows.append(np.sin(2 * np.pi * k * x / n))
        a.append(k)
        m.append(2.0)
    return np.array(rows), np.array(a), np.array(m)


def pool(r, N):
    """2x2x2 average pooling of fields r[..., N2*N1*N0] (x fastest)."""
    lead = r.shape[:-1]
    v = r.reshape(lead + (N[2] // 2, 2, N[1] // 2, 2, N[0] // 2, 2))
    return v.mean(axis=(-5, -3, -1)).reshape(lead + (-1,))


def pool_t(rc, N):
    """Adjoint of pool: replicate each coarse value to its 8 fine points / 8."""
    lead = rc.shape[:-1]
    n = (N[2] // 2, N[1] // 2, N[0] // 2)
    v = rc.reshape(lead + n) / 8.0
    v = np.repeat(np.repeat(np.repeat(v, 2, axis=-3), 2, axis=-2), 2, axis=-1)
    return v.reshape(lead + (-1,))


def features(psi0, V, eps_dd, lam, N):
    """Conditioning fields (NFEAT x coarse points)."""
    dens = pool(np.abs(psi0) ** 2, N)
    vc = pool(np.asarray(V, float), N)
    nc = dens.size
    phi = np.empty((NFEAT, nc))
    phi[0] = 1.0
    phi[1] = dens / max(dens.max(), 1e-300)
    phi[2] = vc / max(np.abs(vc).max(), 1e-300)
    phi[3] = eps_dd
    phi[4] = lam / 4.0
    return phi


class Net:
    """Parameters of S (one half) and eta, with the fixed geometry."""

    def __init__(self, N, C=C_DEF, L=L_DEF, modes=MODES_DEF):
        self.N = list(N)
        self.n = [N[0] // 2, N[1] // 2, N[2] // 2]
        self.C, self.L, self.modes = C, L, modes
        self.E = [basis(self.n[d], modes) for d in range(3)]
        self.R = 2 * modes - 1
        self.A = np.zeros((C, NFEAT))
        self.W = np.zeros((L, C, modes, modes, modes))   # [l][c][az][ay][ax]
        self.B = np.zeros((L, C, C))
        self.Dg = np.zeros((L, C, NFEAT))
        self.eta = 0.0

    # flat parameter vector in the order A, W, B, Dg, eta (the CUDA layout)
    def flat(self):
        return np.concatenate([self.A.ravel(), self.W.ravel(), self.B.ravel(), self.Dg.ravel(), [self.eta]])

    def set_flat(self, v):
        i = 0
        for name in ("A", "W", "B", "Dg"):
            a = getattr(self, name)
            setattr(self, name, np.asarray(v[i:i + a.size], float).reshape(a.shape))
            i += a.size
        self.eta = float(v[i])

    def nparams(self):
        return self.A.size + self.W.size + self.B.size + self.Dg.size + 1

    def wfull(self, l, c):
        """w_l[c] on the R^3 coefficient grid (z, y, x order)."""
        (_, az, mz), (_, ay, my), (_, ax, mx) = self.E[2], self.E[1], self.E[0]
        n3 = self.n[0] * self.n[1] * self.n[2]
        Wl = self.W[l, c]
        return Wl[np.ix_(az, ay, ax)] * (mz[:, None, None] * my[None, :, None] * mx[None, None, :]) / n3

    def P(self, z):
        """z[..., nz*ny*nx] -> coefficients [..., R, R, R]."""
        lead = z.shape[:-1]
        v = z.reshape(lead + (self.n[2], self.n[1], self.n[0]))
        v = np.einsum("...zyx,ix->...zyi", v, self.E[0][0])
        v = np.einsum("...zyi,jy->...zji", v, self.E[1][0])
        v = np.einsum("...zji,kz->...kji", v, self.E[2][0])
        return v

    def Pt(self, c):
        lead = c.shape[:-3]
        v = np.einsum("...kji,kz->...zji", c, self.E[2][0])
        v = np.einsum("...zji,jy->...zyi", v, self.E[1][0])
        v = np.einsum("...zyi,ix->...zyx", v, self.E[0][0])
        return v.reshape(lead + (-1,))

    def sc(self, l, z):
        """SC_l on z[C, nc]."""
        out = np.empty_like(z)
        co = self.P(z)
        for c in range(self.C):
            out[c] = self.Pt(co[c] * self.wfull(l, c))
        return out

    def pm(self, l, z, phi, transpose=False):
        diag = self.Dg[l] @ phi  # [C, nc]
        Bm = self.B[l].T if transpose else self.B[l]
        return Bm @ z + diag * z

    def lift_coef(self, phi):
        return self.A @ phi  # [C, nc]

    def forward(self, r, phi, keep=False):
        """S r for one fine field r; with keep, also the layer inputs."""
        rc = pool(r, self.N)
        z = self.lift_coef(phi) * rc[None, :]
        acts = [z]
        for l in range(self.L):
            z = z + self.sc(l, z) + self.pm(l, z, phi)
            acts.append(z)
        return (z, acts, rc) if keep else z

    def adjoint(self, g, phi):
        """S^T g for g[C, nc]."""
        for l in reversed(range(self.L)):
            g = g + self.sc(l, g) + self.pm(l, g, phi, transpose=True)
        rc = np.sum(self.lift_coef(phi) * g, axis=0)
        return pool_t(rc, self.N)

    def apply(self, r, phi, p0r):
        """T r = S^T S r + exp(eta) P0 r (p0r = P0 r given)."""
        return self.adjoint(self.forward(r, phi), phi) + np.exp(self.eta) * p0r

    def backprop(self, v, u, phi):
        """Gradient (flat, without eta) of <u, S v> with respect to A, W, B, Dg."""
        _, acts, rc = self.forward(v, phi, keep=True)
        gA = np.zeros_like(self.A)
        gW = np.zeros_like(self.W)
        gB = np.zeros_like(self.B)
        gD = np.zeros_like(self.Dg)
        g = u.copy()
        (_, az, mz), (_, ay, my), (_, ax, mx) = self.E[2], self.E[1], self.E[0]
        n3 = self.n[0] * self.n[1] * self.n[2]
        mult = (mz[:, None, None] * my[None, :, None] * mx[None, None, :]) / n3
        for l in reversed(range(self.L)):
            z = acts[l]
            pz = self.P(z)
            pg = self.P(g)
            for c in range(self.C):
                prod = pz[c] * pg[c] * mult
                np.add.at(gW[l, c], np.ix_(az, ay, ax), prod)
            gB[l] += g @ z.T
            gD[l] += (g * z) @ phi.T
            g = g + self.sc(l, g) + self.pm(l, g, phi, transpose=True)
        gA += (g * rc[None, :]) @ phi.T
        return np.concatenate([gA.ravel(), gW.ravel(), gB.ravel(), gD.ravel()])

    def loss_and_grad(self, r, e, p0r, phi):
        """Loss ||T r - e||^2 / ||e||^2 of one pair and its flat gradient."""
        tr = self.apply(r, phi, p0r)
        d = tr - e
        ee = float(e @ e)
        loss = float(d @ d) / ee
        sr = self.forward(r, phi)
        sd = self.forward(d, phi)
        g = (self.backprop(d, sr, phi) + self.backprop(r, sd, phi)) * (2.0 / ee)
        geta = 2.0 * np.exp(self.eta) * float(d @ p0r) / ee
        return loss, np.concatenate([g, [geta]])


def loss_and_grad_energy(net, r, e, p0r, phi, aop):
    """Energy-norm loss of one pair, ||T r - e||_A^2 / ||e||_A^2 with
    e = A^-1 r, evaluated as (<Tr, A Tr> - 2 <r, Tr> + <r, e>) / <r, e>, and
    its gradient: with d = A T r - r it is 2 / <r, e> grad <S d, S r> (d, r
    held fixed) and 2 exp(eta) <d, P0 r> / <r, e> for eta.  aop(x) = A x."""
    tr = net.apply(r, phi, p0r)
    atr = aop(tr)
    re = float(r @ e)
    loss = (float(tr @ atr) - 2.0 * float(r @ tr) + re) / re
    d = atr - r
    sr = net.forward(r, phi)
    sd = net.forward(d, phi)
    g = (net.backprop(d, sr, phi) + net.backprop(r, sd, phi)) * (2.0 / re)
    geta = 2.0 * np.exp(net.eta) * float(d @ p0r) / re
    return loss, np.concatenate([g, [geta]])


def adam(params, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015), in place on params, m, v; step >= 1."""
    m *= b1
    m += (1 - b1) * grad
    v *= b2
    v += (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    params -= lr * mh / (np.sqrt(vh) + eps)
