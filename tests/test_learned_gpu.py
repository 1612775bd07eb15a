"""Learned SPD preconditioner on the GPU (bdg/bdg_learn.h).

* apply, loss, gradient and Adam step of the CUDA kernels against the oracle
  (oracle/learned_precond.py) on a 16^3 grid with random parameters:
  FP32 kernels, so 1e-5 relative on applies and loss, 1e-4 on the gradient;
* T symmetric and positive definite as computed;
* the inner CG reaches its tolerance on (K + sigma) e = r;
* what training gains: on the 32^3 dipolar trap (eps_dd 0.5, nev 8, tol 1e-8
  true residual) a network trained on residuals harvested from the plain
  solve needs fewer iterations than the plain preconditioner, to the same
  eigenvalues (1e-9 relative);
* a network that slows the solve (a large random coarse term added to P0)
  is dropped by the stall fallback and the solve still converges.
"""
import numpy as np
import pytest

from oracle import learned_precond as LP

pytestmark = pytest.mark.gpu

N = [16, 16, 16]
S = 16 ** 3
SHAPE = (4, 2, 3)  # C, L, modes


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


def relerr(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture
def setup(bdg):
    torch = _torch()
    rng = np.random.default_rng(12)
    C_, L_, M_ = SHAPE
    lp = bdg.LearnedPrecond(N, C_, L_, M_)
    lp.set_fast_math(False)  # exact FP32 against the oracle
    psi, V = rng.standard_normal(S), rng.random(S)
    lp.condition(psi, V, 0.6, 2.0)
    nets = []
    for h in range(2):
        net = LP.Net(N, C=C_, L=L_, modes=M_)
        th = (0.2 * rng.standard_normal(net.nparams())).astype(np.float32)
        th[-1] = 0.3
        lp.set_params(h, th)
        net.set_flat(th.astype(np.float64))
        nets.append(net)
    phi = LP.features(psi, V, 0.6, 2.0, N)
    dc = bdg.DeviceContext(3, N, [8.0] * 3, False)
    return torch, lp, nets, phi, dc, rng


def test_apply_matches_oracle(setup, bdg):
    torch, lp, nets, phi, dc, rng = setup
    x = rng.standard_normal((3, S))
    y0 = rng.standard_normal((3, S))
    for prec, tol in ((0, 1e-5), (1, 1e-4)):
        dt = torch.float32 if prec else torch.float64
        for h in range(2):
            xt = torch.tensor(x, dtype=dt, device="cuda")
            yt = torch.tensor(y0, dtype=dt, device="cuda")
            torch.cuda.synchronize()
            lp.apply_half_ptr(dc, h, prec, xt.data_ptr(), S, yt.data_ptr(), S, 3)
            dc.synchronize()
            got = yt.double().cpu().numpy()
            for c in range(3):
                ref = nets[h].apply(x[c], phi, y0[c])
                assert relerr(got[c], ref) < tol, (prec, h, c, relerr(got[c], ref))


def test_t_symmetric_positive(setup, bdg):
    torch, lp, nets, phi, dc, rng = setup
    x, z = rng.standard_normal(S), rng.standard_normal(S)

    def T(v):
        vt = torch.tensor(v[None, :], device="cuda")
        yt = vt.clone()  # P0 = identity
        torch.cuda.synchronize()
        lp.apply_half_ptr(dc, 1, 0, vt.data_ptr(), S, yt.data_ptr(), S, 1)
        dc.synchronize()
        return yt.cpu().numpy()[0]

    tx, tz = T(x), T(z)
    assert abs(tx @ z - x @ tz) < 1e-5 * abs(tx @ z)
    assert tx @ x > 0 and tz @ z > 0


def test_gradient_and_adam_match_oracle(setup, bdg):
    torch, lp, nets, phi, dc, rng = setup
    B = 3
    r, e, p0 = rng.standard_normal((B, S)), rng.standard_normal((B, S)), 0.5 * rng.standard_normal((B, S))
    rt, et, pt = (torch.tensor(a, device="cuda") for a in (r, e, p0))
    torch.cuda.synchronize()
    for h in range(2):
        loss, g = lp.loss_grad(dc, h, rt.data_ptr(), et.data_ptr(), pt.data_ptr(), S, B)
        ls, gs = [], []
        for c in range(B):
            l1, g1 = nets[h].loss_and_grad(r[c], e[c], p0[c], phi)
            ls.append(l1)
            gs.append(g1)
        lref, gref = np.mean(ls), np.mean(gs, axis=0)
        assert abs(loss - lref) < 1e-5 * abs(lref), (loss, lref)
        assert np.linalg.norm(g - gref) < 1e-4 * np.linalg.norm(gref), np.linalg.norm(g - gref) / np.linalg.norm(gref)
        # one Adam step from zero moments: p - lr * g / (|g| + eps)
        before = lp.get_params(h).astype(np.float64)
        lp.set_params(h, before.astype(np.float32))  # resets the moments
        lp.train_step(dc, h, rt.data_ptr(), et.data_ptr(), pt.data_ptr(), S, B, 1e-3)
        after = lp.get_params(h).astype(np.float64)
        th = before.copy()
        LP.adam(th, g.astype(np.float64), np.zeros_like(th), np.zeros_like(th), 1, 1e-3)
        assert np.max(np.abs(after - th)) < 1e-6


def test_energy_gradient_matches_oracle(setup, bdg):
    """Energy-norm loss of A = K + sigma through the library's K apply,
    against the oracle with its own K (same fields)."""
    from oracle import bdg_oracle as O

    torch, lp, nets, phi, _, rng = setup
    sigma = 0.8
    ltK = 1 + rng.random(S)
    dc = bdg.DeviceContext(3, N, [8.0] * 3, False)
    dc.set_fields(ltK=ltK, ltM=2 + rng.random(S), wf=rng.standard_normal(S), pK=0.5 + rng.random(S),
                  pM=0.5 + rng.random(S), mu=0.5, vdd=np.zeros((N[0] // 2 + 1) * 256), g_ddi=0.0, dipolar=False)
    oc = O.Ctx(3, N, [8.0] * 3, False)
    O.set_system(oc)
    oc.localTermK = ltK.copy()
    B = 3
    r, p0 = rng.standard_normal((B, S)), 0.5 * rng.standard_normal((B, S))
    rt, pt = torch.tensor(r, device="cuda"), torch.tensor(p0, device="cuda")
    et = torch.zeros_like(rt)
    torch.cuda.synchronize()
    bdg.lp_cg(dc, bdg.OP_K, sigma, rt.data_ptr(), et.data_ptr(), S, B, 1e-13, 2000)
    e = et.cpu().numpy()
    lp.set_energy_loss(sigma)
    loss, g = lp.loss_grad(dc, 0, rt.data_ptr(), et.data_ptr(), pt.data_ptr(), S, B)
    lp.set_energy_loss(-1.0)
    ls, gs = [], []
    for c in range(B):
        l1, g1 = LP.loss_and_grad_energy(nets[0], r[c], e[c], p0[c], phi, lambda x: O.matmulK(oc, x) + sigma * x)
        ls.append(l1)
        gs.append(g1)
    lref, gref = np.mean(ls), np.mean(gs, axis=0)
    assert abs(loss - lref) < 1e-5 * abs(lref), (loss, lref)
    assert np.linalg.norm(g - gref) < 1e-4 * np.linalg.norm(gref), np.linalg.norm(g - gref) / np.linalg.norm(gref)


def test_cg_solves_shifted_k(bdg):
    torch = _torch()
    rng = np.random.default_rng(5)
    dc = bdg.DeviceContext(3, N, [8.0] * 3, False)
    dc.set_fields(ltK=1 + rng.random(S), ltM=2 + rng.random(S), wf=rng.standard_normal(S), pK=0.5 + rng.random(S),
                  pM=0.5 + rng.random(S), mu=0.5, vdd=rng.standard_normal((N[0] // 2 + 1) * 256), g_ddi=0.1,
                  dipolar=False)
    r = torch.tensor(rng.standard_normal((4, S)), device="cuda")
    e = torch.zeros_like(r)
    torch.cuda.synchronize()
    it = bdg.lp_cg(dc, bdg.OP_K, 0.7, r.data_ptr(), e.data_ptr(), S, 4, 1e-10, 500)
    ke = torch.zeros_like(r)
    dc.apply_ptr(bdg.OP_K, 0, e.data_ptr(), S, ke.data_ptr(), S, 4)
    dc.synchronize()
    res = (ke + 0.7 * e - r).norm(dim=1) / r.norm(dim=1)
    assert it > 0 and float(res.max()) < 1e-9


def _c1(B):
    from bdg_lobpcg_b200 import problems

    cfg = problems.config(32)
    psi, mu, _, _, V = problems.ground_state(B, cfg)
    return problems, cfg, psi, mu, V


def test_training_gains_iterations(bdg):
    """Trained on the plain solve's own residuals, the learned T converges in
    fewer iterations than the plain preconditioner, to the same spectrum."""
    _torch()
    from bdg_lobpcg_b200 import learn

    problems, cfg, psi, mu, V = _c1(bdg)
    p, _ = problems.build(bdg, cfg, psi, mu, V, "f64")
    pairs, it_plain = learn.make_pairs(bdg, p, cfg, psi, V, cap=600, sigma=1.0)
    lam_plain = p.eigenvalues().copy()
    dev = p.device_context()
    lp = bdg.LearnedPrecond(cfg["N"], 16, 4, 4)
    lp.init_random(0.05, 4)
    lp.condition(psi, V, cfg["eps_dd"], cfg["lam"])
    lp.set_energy_loss(1.0)
    before = learn.eval_loss(lp, dev, pairs)
    learn.train(lp, dev, pairs, steps=3000, batch=16, lr=2e-3, seed=0, cosine=True)
    after = learn.eval_loss(lp, dev, pairs)
    p.close()
    for h in (0, 1):
        assert after[h] < before[h], (h, before, after)
    it_l, _, lam_l, tres, fb, _ = learn.solve_with(bdg, cfg, psi, mu, V, lp)
    assert tres <= cfg["tol"]
    assert np.max(np.abs(lam_l - lam_plain) / np.abs(lam_plain)) < 1e-9
    assert it_l < it_plain, (it_l, it_plain, fb, before, after)


def test_stall_falls_back_to_plain(bdg):
    _torch()
    from bdg_lobpcg_b200 import learn

    problems, cfg, psi, mu, V = _c1(bdg)
    lp = bdg.LearnedPrecond(cfg["N"], 4, 2, 4)
    rng = np.random.default_rng(9)
    for h in range(2):
        th = np.zeros(lp.nparams, dtype=np.float32)
        th[: 4 * 5] = 30.0 * rng.standard_normal(4 * 5)  # a large random coarse term on top of P0
        lp.set_params(h, th)
    lp.condition(psi, V, cfg["eps_dd"], cfg["lam"])
    it, _, lam, tres, fb, _ = learn.solve_with(bdg, cfg, psi, mu, V, lp, stall_window=4)
    assert fb >= 0, (it, fb)
    assert tres <= cfg["tol"]
