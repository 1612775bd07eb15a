"""Batched sweep of independent BdG problems (the benchmark's batching case).

    python -m bdg_lobpcg_b200.sweep [--problems 64] [--concurrency 8] [--graphs 1] [--seed 3]

64 real problems with grids drawn uniformly from {32, 48, 64, 96}^3, box
half-width 1.5 R_TF, eps_dd ~ U[0, 0.9], lambda ~ U[0.5, 4], g ~ U[200, 2000]
(seed 3); nev 16, sizeSub 32, tol 1e-8 on the true residual, Goldstone
deflation, X0 ~ N(0, 1) with v = u.  Ground states come from the GPU
producer (set-up, not timed).  The problems are solved twice: one after the
other (bdg_solve, plain), then together through bdg_solve_batch
(`concurrency` solves in flight, operator applies replayed as CUDA graphs),
and the script prints one JSON line with the aggregate solves per second of
both, the per-problem wall times and the largest eigenvalue difference
between the two runs.

R_TF is the Thomas-Fermi radius of the contact problem along the weakest
trap axis: mu_TF = (15 g lambda / (4 pi))^(2/5) / 2 for the trap
(1, 1, lambda) and a unit-norm condensate, R = sqrt(2 mu_TF) / min(1, lambda).
"""
import argparse
import json
import math
import sys
import time

import numpy as np

from . import problems


def sweep_configs(n, seed=3, nev=16):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        grid = int(rng.choice([32, 48, 64, 96]))
        eps = float(rng.uniform(0.0, 0.9))
        lam = float(rng.uniform(0.5, 4.0))
        g = float(rng.uniform(200.0, 2000.0))
        mu_tf = 0.5 * (15.0 * g * lam / (4.0 * math.pi)) ** 0.4
        R = math.sqrt(2.0 * mu_tf) / min(1.0, lam)
        box = 2.0 * 1.5 * R
        cfg = problems.config(grid, eps_dd=eps, lam=lam, g=g, nev=nev, seed=int(rng.integers(1 << 30)), box=box)
        cfg["rc"] = 0.5 * box
        out.append(cfg)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--problems", type=int, default=64)
    ap.add_argument("--concurrency", type=int, default=8)
    ap.add_argument("--graphs", type=int, default=1)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--nev", type=int, default=16)
    a = ap.parse_args(argv)
    import bdg_lobpcg_b200 as B

    cfgs = sweep_configs(a.problems, a.seed, a.nev)
    t0 = time.perf_counter()
    states = [problems.ground_state(B, c) for c in cfgs]
    t_gs = time.perf_counter() - t0

    def build_all():
        out = []
        for c, (psi, mu, _, _, V) in zip(cfgs, states):
            p, _ = problems.build(B, c, psi, mu, V, "f64")
            out.append(p)
        return out

    # one after the other
    probs = build_all()
    seq_t = np.zeros(len(probs))
    seq_it = []
    seq_eigs = []
    t0 = time.perf_counter()
    for i, p in enumerate(probs):
        s0 = time.perf_counter()
        rc = p.solve()
        seq_t[i] = time.perf_counter() - s0
        if rc:
            raise RuntimeError(f"problem {i}: solve failed ({rc})")
        seq_it.append(p.stats()["iterations"])
        seq_eigs.append(p.eigenvalues().copy())
        B.lib().bdg_release_device_memory(p._h)
    t_seq = time.perf_counter() - t0
    for p in probs:
        p.close()
    # batched
    probs = build_all()
    t0 = time.perf_counter()
    rcs, bat_t = B.solve_batch(probs, concurrency=a.concurrency, graphs=bool(a.graphs))
    t_bat = time.perf_counter() - t0
    if any(rcs):
        raise RuntimeError(f"batched solves failed: {rcs}")
    diff = max(float(np.max(np.abs(p.eigenvalues() - e) / np.abs(e))) for p, e in zip(probs, seq_eigs))
    bat_it = [p.stats()["iterations"] for p in probs]
    tres = max(p.stats()["max_true_residual"] for p in probs)
    for p in probs:
        p.close()
    grids = [c["N"][0] for c in cfgs]
    print(json.dumps({
        "problems": len(cfgs), "grids": {str(g): grids.count(g) for g in sorted(set(grids))},
        "nev": a.nev, "concurrency": a.concurrency, "graphs": bool(a.graphs),
        "sequential": {"seconds": t_seq, "solves_per_s": len(cfgs) / t_seq, "per_problem_s": seq_t.tolist(),
                       "iterations": seq_it},
        "batched": {"seconds": t_bat, "solves_per_s": len(cfgs) / t_bat, "per_problem_s": bat_t.tolist(),
                    "iterations": bat_it},
        "speedup": t_seq / t_bat, "max_rel_eig_diff": diff, "max_true_residual": tres,
        "ground_states_s": t_gs}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
