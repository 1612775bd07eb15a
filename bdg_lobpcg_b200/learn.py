"""Training-pair generation and training of the learned preconditioner.

    python -m bdg_lobpcg_b200.learn train --out precond.bin [--problems 16] [--grid 64] ...
    python -m bdg_lobpcg_b200.learn eval --model precond.bin [--grid 128] [--eps 0.85,0.9]

Pairs (r, e) come from the solver itself: the residual columns R = A X -
lambda B X of plain FP64 solves are harvested on the device
(bdg_set_residual_harvest); each half gives a pair for its network, with
e = (K + sigma)^-1 r_u or (M + sigma)^-1 r_v from the library's inner CG
(bdg_lp_cg) and P0 r from the plain preconditioner (T_K, T_M).  Columns are
scaled to unit residual norm (the loss is scale invariant).  The loss is the
energy norm ||T r - e||_A^2 / ||e||_A^2 of A = Op + sigma (the norm in
which a preconditioner's quality shows in the eigensolver; fitting e in
the plain 2-norm made the solver slower).  Training runs the library's
forward / adjoint / gradient / Adam kernels (bdg_lp_train_step) on random
batches.  torch only holds device buffers.

The sweep of the benchmark's learned-preconditioner configuration: 64^3
problems in [-12, 12)^3 with eps_dd ~ U[0, 0.8], lambda ~ U[0.5, 3],
g = 1000 (seed 4); evaluation on held-out 128^3 problems, eps_dd in
{0.85, 0.9}, lambda = 2, nev 32, tol 1e-8, against the plain preconditioner.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import problems


def _torch():
    import torch

    return torch


def make_pairs(B, p, cfg, psi, V, cap, sigma=1.0, cg_tol=1e-6, cg_maxit=400, maxiter=None):
    """Harvest up to `cap` residual columns from a plain solve of Problem p and
    turn them into training pairs for both halves.  Returns
    {half: (r, e, p0r)} (torch FP64 [ncol, S] each) and the solve's iterations."""
    torch = _torch()
    S = int(np.prod(cfg["N"]))
    n = 2 * S
    buf = torch.zeros(cap, n, dtype=torch.float64, device="cuda")
    p.set_residual_harvest(buf.data_ptr(), cap)
    if maxiter is not None:
        p.set_solver_params(cfg["nev"], cfg["sizeSub"], maxiter, cfg["tol"])
    rc = p.solve()
    if rc:
        raise RuntimeError(f"harvest solve failed ({rc})")
    iters = p.stats()["iterations"]
    cnt = p.residual_harvest_count()
    p.set_residual_harvest(0, 0)
    torch.cuda.synchronize()
    R = buf[:cnt]
    dev = p.device_context()
    out = {}
    for half, op, top in ((0, B.OP_K, B.OP_TK), (1, B.OP_M, B.OP_TM)):
        r = R[:, half * S:(half + 1) * S].contiguous()
        nr = torch.linalg.vector_norm(r, dim=1, keepdim=True).clamp_min(1e-300)
        r = r / nr
        e = torch.zeros_like(r)
        p0 = torch.zeros_like(r)
        torch.cuda.synchronize()
        B.lp_cg(dev, op, sigma, r.data_ptr(), e.data_ptr(), S, r.shape[0], cg_tol, cg_maxit)
        dev.apply_ptr(top, 0, r.data_ptr(), S, p0.data_ptr(), S, r.shape[0])
        dev.synchronize()
        out[half] = (r, e, p0)
    return out, iters


def train(lp, dev, pairs, steps=300, batch=16, lr=1e-3, seed=0, log=None, cosine=False, t0=0, total=None):
    """Adam on random batches of the pairs of each half (cosine: learning
    rate lr * (1 + cos(pi t / total)) / 2 at global step t = t0 + it, total
    defaulting to steps); returns the loss history {half: [(step, loss)]}."""
    import math

    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = {}
    for half, (r, e, p0) in pairs.items():
        S = r.shape[1]
        hist[half] = []
        ncol = r.shape[0]
        for it in range(steps):
            idx = torch.randint(0, ncol, (min(batch, ncol),), generator=g).cuda()
            rb, eb, pb = r[idx].contiguous(), e[idx].contiguous(), p0[idx].contiguous()
            torch.cuda.synchronize()
            T = total if total else steps
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * min(t0 + it, T) / T)) if cosine else lr
            loss = lp.train_step(dev, half, rb.data_ptr(), eb.data_ptr(), pb.data_ptr(), S, rb.shape[0], lr_t)
            hist[half].append((it, loss))
            if log and (it % 50 == 0 or it == steps - 1):
                log(f"half {half} step {it} loss {loss:.5f}")
    return hist


def eval_loss(lp, dev, pairs):
    """Mean loss of each half over all pairs (no update)."""
    torch = _torch()
    out = {}
    for half, (r, e, p0) in pairs.items():
        torch.cuda.synchronize()
        tot, cnt = 0.0, 0
        for c0 in range(0, r.shape[0], 32):
            rb, eb, pb = r[c0:c0 + 32], e[c0:c0 + 32], p0[c0:c0 + 32]
            loss, _ = lp.loss_grad(dev, half, rb.data_ptr(), eb.data_ptr(), pb.data_ptr(), r.shape[1], rb.shape[0],
                                   want_grad=False)
            tot += loss * rb.shape[0]
            cnt += rb.shape[0]
        out[half] = tot / max(cnt, 1)
    return out


def solve_with(B, cfg, psi, mu, V, lp=None, precision="f64", stall_window=0):
    """Fresh problem, same X0; returns (iterations, seconds, eigenvalues,
    max true residual, fallback iteration, device seconds)."""
    p, _ = problems.build(B, cfg, psi, mu, V, precision)
    if lp is not None:
        p.set_learned_precond(lp, stall_window)
    t0 = time.perf_counter()
    rc = p.solve()
    t = time.perf_counter() - t0
    if rc:
        raise RuntimeError(f"solve failed ({rc})")
    st = p.stats()
    res = (st["iterations"], t, p.eigenvalues().copy(), st["max_true_residual"],
           p.learned_fallback_iteration() if lp is not None else -1, st["seconds_device"])
    p.close()
    return res


def cmd_train(a):
    import bdg_lobpcg_b200 as B

    rng = np.random.default_rng(a.seed)
    lp = None
    t0 = time.perf_counter()
    npairs = 0
    for k in range(a.problems):
        eps = float(rng.uniform(0.0, 0.8))
        lam = float(rng.uniform(0.5, 3.0))
        cfg = problems.config(a.grid, eps_dd=eps, lam=lam, nev=a.nev, seed=int(rng.integers(1 << 30)))
        psi, mu, _, _, V = problems.ground_state(B, cfg)
        p, _ = problems.build(B, cfg, psi, mu, V, "f64", maxiter=a.harvest_iters)
        if lp is None:
            lp = B.LearnedPrecond(cfg["N"], a.channels, a.layers, a.modes)
            lp.init_random(a.init_amp, a.seed)
        pairs, iters = make_pairs(B, p, cfg, psi, V, a.cap, sigma=a.sigma)
        lp.condition(psi, V, eps, lam)
        lp.set_energy_loss(a.sigma)
        dev = p.device_context()
        hist = train(lp, dev, pairs, steps=a.steps, batch=a.batch, lr=a.lr, seed=k, cosine=True, t0=k * a.steps,
                     total=a.problems * a.steps)
        npairs += 2 * pairs[0][0].shape[0]
        print(json.dumps({"problem": k, "eps_dd": eps, "lambda": lam, "mu": mu, "harvest_iters": iters,
                          "pairs": 2 * pairs[0][0].shape[0], "loss_K": hist[0][-1][1], "loss_M": hist[1][-1][1],
                          "seconds": time.perf_counter() - t0}), flush=True)
        p.close()
    lp.save(a.out)
    print(json.dumps({"saved": a.out, "pairs": npairs, "seconds": time.perf_counter() - t0}))
    return 0


def cmd_eval(a):
    import bdg_lobpcg_b200 as B

    lp = None
    for eps in [float(v) for v in a.eps.split(",")]:
        cfg = problems.config(a.grid, eps_dd=eps, lam=a.lam, nev=a.nev, seed=4)
        psi, mu, _, _, V = problems.ground_state(B, cfg)
        if lp is None:
            lp = B.LearnedPrecond(cfg["N"], a.channels, a.layers, a.modes)
            lp.load(a.model)
        lp.condition(psi, V, eps, a.lam)
        plain = solve_with(B, cfg, psi, mu, V, None, a.precision)
        learned = solve_with(B, cfg, psi, mu, V, lp, a.precision)
        rel = float(np.max(np.abs(learned[2] - plain[2]) / np.abs(plain[2])))
        print(json.dumps({"grid": a.grid, "eps_dd": eps, "lambda": a.lam, "nev": cfg["nev"],
                          "plain": {"iterations": plain[0], "seconds": plain[1], "device_s": plain[5],
                                    "max_true_residual": plain[3]},
                          "learned": {"iterations": learned[0], "seconds": learned[1], "device_s": learned[5],
                                      "max_true_residual": learned[3], "fallback_iteration": learned[4]},
                          "max_rel_eig_diff": rel}), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    t.add_argument("--problems", type=int, default=16)
    t.add_argument("--grid", type=int, default=64)
    t.add_argument("--nev", type=int, default=16)
    t.add_argument("--cap", type=int, default=512)
    t.add_argument("--harvest-iters", type=int, default=60)
    t.add_argument("--steps", type=int, default=1000)
    t.add_argument("--batch", type=int, default=16)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--sigma", type=float, default=1.0)
    t.add_argument("--init-amp", type=float, default=0.05)
    t.add_argument("--seed", type=int, default=4)
    for q in (t,):
        q.add_argument("--channels", type=int, default=16)
        q.add_argument("--layers", type=int, default=4)
        q.add_argument("--modes", type=int, default=12)
    e = sub.add_parser("eval")
    e.add_argument("--model", required=True)
    e.add_argument("--grid", type=int, default=128)
    e.add_argument("--nev", type=int, default=32)
    e.add_argument("--eps", default="0.85,0.9")
    e.add_argument("--lam", type=float, default=2.0)
    e.add_argument("--precision", default="f64")
    e.add_argument("--channels", type=int, default=16)
    e.add_argument("--layers", type=int, default=4)
    e.add_argument("--modes", type=int, default=12)
    a = ap.parse_args(argv)
    return cmd_train(a) if a.cmd == "train" else cmd_eval(a)


if __name__ == "__main__":
    sys.exit(main())
