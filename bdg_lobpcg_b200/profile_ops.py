"""Run a fixed number of batched operator applies for profiling (ncu).

    python -m bdg_lobpcg_b200.profile_ops [--grid 128] [--ncol 8] [--prec 0|1] [--reps 3]

Random fields and columns on a grid^3 dipolar context; applies LREP and TLREP
`reps` times each (after one warm-up apply), then a Gram of the block.
"""
import argparse
import sys

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--ncol", type=int, default=8)
    ap.add_argument("--prec", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    import torch

    import bdg_lobpcg_b200 as B

    N = [a.grid] * 3
    S = a.grid ** 3
    H = (a.grid // 2 + 1) * a.grid * a.grid
    rng = np.random.default_rng(0)
    dc = B.DeviceContext(3, N, [24.0] * 3, False)
    dc.set_fields(ltK=1 + rng.random(S), ltM=2 + rng.random(S), wf=rng.random(S), pK=rng.random(S) + 0.5,
                  pM=rng.random(S) + 0.5, mu=1.0, vdd=rng.standard_normal(H), g_ddi=0.5, dipolar=True)
    dt = torch.float32 if a.prec else torch.float64
    x = torch.randn(a.ncol, 2 * S, dtype=dt, device="cuda")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    for op in (B.OP_LREP, B.OP_TLREP):
        for _ in range(1 + a.reps):
            dc.apply_ptr(op, a.prec, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, a.ncol)
    out = torch.zeros(4 * a.ncol * a.ncol, dtype=torch.float64, device="cuda")
    dc.gram_ptr(a.prec, False, S, a.ncol, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, out.data_ptr())
    dc.synchronize()
    print("profile_ops done", a)
    return 0


if __name__ == "__main__":
    sys.exit(main())
