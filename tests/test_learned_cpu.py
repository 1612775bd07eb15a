"""The oracle of the learned preconditioner pinned by its own algebra.

The learned preconditioner has no counterpart in the reference, so its
checker (oracle/learned_precond.py) is pinned by what the construction
guarantees: S^T is the adjoint of S, T = S^T S + exp(eta) P0 is symmetric
and positive definite, the spectral convolution equals an FFT filter with an
even transfer function, and the analytic gradient of the loss matches
central finite differences.  Small grids (8^3 fine, 4^3 coarse, 2 modes).
"""
import numpy as np
import pytest

from oracle import learned_precond as LP

N = [8, 8, 8]


def _net(seed, C=3, L=2, modes=2):
    rng = np.random.default_rng(seed)
    net = LP.Net(N, C=C, L=L, modes=modes)
    net.set_flat(0.3 * rng.standard_normal(net.nparams()))
    return net, rng


def _phi(rng):
    S = int(np.prod(N))
    return LP.features(rng.standard_normal(S), rng.random(S), 0.6, 2.0, N)


def test_adjoint_and_symmetry():
    net, rng = _net(1)
    phi = _phi(rng)
    S = int(np.prod(N))
    x, y = rng.standard_normal(S), rng.standard_normal(S)
    g = rng.standard_normal((net.C, S // 8))
    # <S x, g> = <x, S^T g>
    assert abs(np.sum(net.forward(x, phi) * g) - x @ net.adjoint(g, phi)) < 1e-10 * abs(x @ net.adjoint(g, phi)) + 1e-12
    # T symmetric and positive with P0 = identity
    tx, ty = net.apply(x, phi, x), net.apply(y, phi, y)
    assert abs(tx @ y - x @ ty) < 1e-10 * abs(tx @ y)
    assert tx @ x > 0


def test_spectral_conv_is_even_fft_filter():
    """SC(z) = ifftn(G * fftn(z)) with G(k) = W[|kz|, |ky|, |kx|] on |k_i| < modes."""
    net, rng = _net(2, C=1, L=1, modes=2)
    n = net.n
    z = rng.standard_normal((1, n[0] * n[1] * n[2]))
    got = net.sc(0, z)[0].reshape(n[2], n[1], n[0])
    G = np.zeros((n[2], n[1], n[0]))
    for kz in range(n[2]):
        for ky in range(n[1]):
            for kx in range(n[0]):
                a = [min(k, m - k) for k, m in ((kz, n[2]), (ky, n[1]), (kx, n[0]))]
                if max(a) < net.modes:
                    G[kz, ky, kx] = net.W[0, 0, a[0], a[1], a[2]]
    ref = np.real(np.fft.ifftn(G * np.fft.fftn(z[0].reshape(n[2], n[1], n[0]))))
    assert np.max(np.abs(got - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_gradient_matches_finite_differences():
    net, rng = _net(3)
    phi = _phi(rng)
    S = int(np.prod(N))
    r, e, p0r = rng.standard_normal(S), rng.standard_normal(S), 0.5 * rng.standard_normal(S)
    loss, grad = net.loss_and_grad(r, e, p0r, phi)
    theta = net.flat()
    idx = rng.choice(theta.size, 40, replace=False).tolist() + [theta.size - 1]
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        net.set_flat(tp)
        lp, _ = net.loss_and_grad(r, e, p0r, phi)
        net.set_flat(tm)
        lm, _ = net.loss_and_grad(r, e, p0r, phi)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - grad[i]) < 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])
    net.set_flat(theta)


def test_adam_reduces_loss():
    net, rng = _net(4)
    net.set_flat(np.zeros(net.nparams()))
    net.A[:] = 0.1
    phi = _phi(rng)
    S = int(np.prod(N))
    pairs = [(rng.standard_normal(S), None) for _ in range(4)]
    # targets: a fixed smooth SPD map of r (pooled-and-replicated plus identity)
    pairs = [(r, 2.0 * LP.pool_t(LP.pool(r, N), N) * 8 + 0.3 * r) for r, _ in pairs]
    th = net.flat()
    m, v = np.zeros_like(th), np.zeros_like(th)
    first = None
    for step in range(1, 61):
        g = np.zeros_like(th)
        tot = 0.0
        for r, e in pairs:
            l, gi = net.loss_and_grad(r, e, r, phi)
            tot += l
            g += gi
        first = tot if first is None else first
        LP.adam(th, g / len(pairs), m, v, step, 0.02)
        net.set_flat(th)
    assert tot < 0.5 * first


def test_energy_gradient_matches_finite_differences():
    net, rng = _net(5)
    phi = _phi(rng)
    S = int(np.prod(N))
    dA = 1.0 + rng.random(S)

    def aop(x):  # SPD: positive diagonal plus a smoothing term
        return dA * x + LP.pool_t(LP.pool(x, N), N)

    r, p0r = rng.standard_normal(S), 0.5 * rng.standard_normal(S)
    Am = np.stack([aop(c) for c in np.eye(S)], axis=1)
    e = np.linalg.solve(Am, r)
    loss, grad = LP.loss_and_grad_energy(net, r, e, p0r, phi, aop)
    tr = net.apply(r, phi, p0r)
    assert abs(loss - (tr - e) @ Am @ (tr - e) / (e @ Am @ e)) < 1e-9 * max(loss, 1.0)
    theta = net.flat()
    h = 1e-6
    for i in rng.choice(theta.size, 30, replace=False).tolist() + [theta.size - 1]:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        net.set_flat(tp)
        lp_, _ = LP.loss_and_grad_energy(net, r, e, p0r, phi, aop)
        net.set_flat(tm)
        lm_, _ = LP.loss_and_grad_energy(net, r, e, p0r, phi, aop)
        fd = (lp_ - lm_) / (2 * h)
        assert abs(fd - grad[i]) < 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])
    net.set_flat(theta)
