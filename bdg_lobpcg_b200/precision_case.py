"""Plain FP64 against the mixed FP32/FP64 form on the real (_d) 64^3 and 128^3 problems.

    python -m bdg_lobpcg_b200.precision_case [--grids 64,128] [--steps 1]

Physics: box [-12, 12)^3, trap (1, 1, 2), g = 1000, eps_dd = 0.7, dipoles
along z, cutoff 8; nev 16 at 64^3 and 32 at 128^3 (sizeSub 2 nev), tol 1e-8
on the true residual, Goldstone chain deflated, X0 ~ N(0, 1) at seed 1 with
v = u.  Both forms start from the same psi0 and the same block.  For each
grid the script prints one JSON line: per form the iterations (and FP64
refinement iterations of the mixed form), device and end-to-end seconds,
the largest true residual, and the per-eigenvalue relative difference of
the mixed form from the FP64 form.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import problems


def solve_form(B, cfg, psi, mu, V, prec, steps):
    p, _ = problems.build(B, cfg, psi, mu, V, prec)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        rc = p.solve()
        times.append(time.perf_counter() - t)
        if rc:
            raise RuntimeError(f"{prec} solve failed ({rc})")
    st = p.stats()
    out = {"iterations": st["iterations"], "refine_iterations": st["refine_iterations"],
           "converged": p.converged(), "device_s": st["seconds_device"], "e2e_s": float(np.min(times)),
           "max_true_residual": st["max_true_residual"],
           "stage_ms": {k: st[k] for k in ("ms_apply_A", "ms_apply_T", "ms_residual", "ms_gram", "ms_small_dense",
                                           "ms_update")}}
    ev = p.eigenvalues().copy()
    p.close()
    return out, ev


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grids", default="64,128")
    ap.add_argument("--steps", type=int, default=1)
    a = ap.parse_args(argv)
    import bdg_lobpcg_b200 as B

    for grid in [int(s) for s in a.grids.split(",")]:
        cfg = problems.config(grid)
        psi, mu, _, stat, V = problems.ground_state(B, cfg)
        f64, e64 = solve_form(B, cfg, psi, mu, V, "f64", a.steps)
        mix, emx = solve_form(B, cfg, psi, mu, V, "mixed", a.steps)
        rel = np.abs(emx - e64) / np.abs(e64)
        print(json.dumps({
            "case": f"real _d {grid}^3, FP64 vs mixed FP32/FP64", "grid": cfg["N"], "nev": cfg["nev"],
            "psi0_stationarity": stat, "f64": f64, "mixed": mix,
            "speedup_device": f64["device_s"] / mix["device_s"],
            "max_rel_eig_diff_mixed_vs_f64": float(rel.max()), "rel_eig_diff_mixed_vs_f64": rel.tolist(),
            "eigenvalues_f64": e64.tolist()}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
