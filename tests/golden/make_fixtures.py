"""Generate the ground-state fixtures of the GPU parity tests and of the
32^3 benchmark config (committed as .npz next to this script).

Each psi0 comes from the oracle's split-step imaginary-time propagation
(oracle/bdg_oracle.py: itp_ground_state): unit Gaussian start, dt = 1e-3,
stopped when the per-step change of mu = <psi|H|psi> is below 1e-12,
normalised to sum |psi|^2 dV = 1 on the grid x_i = (i - N/2) L / N.  The
ITP state carries the O(dt^2) splitting error of the time stepping
(||H psi - mu psi|| ~ 1e-3 here); it is then polished by bordered Newton
steps (newton_polish) to the exact discrete stationary state, so that
K psi0 = 0 to ~1e-14 and the Goldstone mode is exact.

    python tests/golden/make_fixtures.py [name ...]
    python tests/golden/make_fixtures.py solve <name> <nev> <seed> [threads]
    python tests/golden/make_fixtures.py solve_config <grid> <psi.npz> [threads]
"""
import os

# OpenBLAS worker threads otherwise spin between BLAS calls and starve the
# OpenMP threads of the reference's CPU FFT (3x slower iterations on 8 cores);
# read when the library loads, so set before numpy / scipy are imported
os.environ.setdefault("OPENBLAS_THREAD_TIMEOUT", "4")
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import bdg_oracle as O  # noqa: E402

# name: (N, L, trap frequencies (x, y, z), g, g_dd, cutoff radius)
PROBLEMS = {
    # small dipolar trap for solver parity tests
    "gs16": ([16, 16, 16], [8.0, 8.0, 8.0], (1.0, 1.0, 2.0), 100.0, 40.0, 4.0),
    # dipolar trap of the 32^3 benchmark config: box [-8, 8)^3, lambda = 2,
    # g = 1000, eps_dd = 0.5, dipoles along z, R_c = 8
    "c1_32": ([32, 32, 32], [16.0, 16.0, 16.0], (1.0, 1.0, 2.0), 1000.0, 500.0, 8.0),
    # the 64^3 grid of the mixed-precision config: box [-12, 12)^3,
    # lambda = 2, g = 1000, eps_dd = 0.7, R_c = 8
    "c2_64": ([64, 64, 64], [24.0, 24.0, 24.0], (1.0, 1.0, 2.0), 1000.0, 700.0, 8.0),
}


def make(name):
    N, L, om, g, gdd, rc = PROBLEMS[name]
    t = time.time()
    psi, mu_itp, steps = O.itp_ground_state(N, L, om, g, gdd, (0.0, 0.0, 1.0), rc, dt=1e-3, tol=1e-12)
    psi, mu, res = O.newton_polish(N, L, om, g, gdd, psi, rc)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), psi=psi, mu=mu, mu_itp=mu_itp, steps=steps,
                        stationarity=res, N=N, L=L, omegas=om, g=g, gdd=gdd, rc=rc)
    print(name, "mu_itp", mu_itp, "mu", mu, "|H psi - mu psi|", res, "steps", steps, "%.1fs" % (time.time() - t))


def solve(name, nev, seed, threads=None):
    """The FP64 CPU oracle solve of fixture `name` through the reference's
    own solve path (oracle/_ref: bdg_solve -> src/solver.c -> restated
    iLOBPCG on the reference operators): nev modes, sizeSub 2 nev, initial
    block X0 ~ N(0, 1) with v = u at `seed`, true residual <= 1e-8, Goldstone
    chain deflated.  Writes <name>_solve.npz: eigenvalues, iterations, the
    per-iteration wall clock and the thread count."""
    from oracle import ref as R

    d = load(name)
    N = [int(v) for v in d["N"]]
    L = [float(v) for v in d["L"]]
    om = [float(v) for v in d["omegas"]]
    m = 2 * nev
    threads = threads or os.cpu_count() or 1
    R.set_threads(threads)
    rp = R.build_problem(N, L, om, float(d["g"]), float(d["gdd"]), d["psi"], float(d["mu"]), Rc=float(d["rc"]))
    size = int(np.prod(N))
    u = np.random.default_rng(seed).standard_normal((m, size))
    rp.set_solver_params(nev, m, 2000, 1e-8)
    rp.set_initial_block(np.concatenate([u, u], axis=1))
    t = time.time()
    res = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    np.savez_compressed(os.path.join(HERE, f"{name}_solve.npz"), eigvals=res["eigvals"], iterations=res["iterations"],
                        converged=res["converged"], timeline=res["timeline"], nev=nev, sizeSub=m, seed=seed,
                        threads=threads)
    print(name, "solve", res["iterations"], "iterations", res["converged"], "converged", "%.1fs" % (time.time() - t))
    print(res["eigvals"])


def solve_config(grid, psi_file, threads=None):
    """The FP64 reference-path solve of the benchmark configuration at
    `grid`^3 (bdg_lobpcg_b200.problems.config) from the psi0 in `psi_file`
    (an .npz with psi and mu from the library's GPU ground-state producer,
    the same psi0 the benchmark computes): writes c2_<grid>_solve.npz with
    the eigenvalues, iterations to tolerance, per-iteration wall clock and the
    psi0's mu and norms, by which bench.py recognises its input."""
    from bdg_lobpcg_b200 import problems
    from oracle import ref as R

    cfg = problems.config(grid)
    d = np.load(psi_file)
    psi, mu = d["psi"], float(d["mu"])
    threads = threads or os.cpu_count() or 1
    R.set_threads(threads)
    V = problems.trap(cfg["N"], cfg["L"], cfg["omegas"])
    rp = R.build_problem(cfg["N"], cfg["L"], cfg["omegas"], cfg["g"], cfg["gdd"], psi, mu, V=V, Rc=cfg["rc"])
    size = int(np.prod(cfg["N"]))
    u = np.random.default_rng(cfg["seed"]).standard_normal((cfg["sizeSub"], size))
    rp.set_solver_params(cfg["nev"], cfg["sizeSub"], 2000, cfg["tol"])
    rp.set_initial_block(np.concatenate([u, u], axis=1))
    t = time.time()
    res = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    np.savez_compressed(os.path.join(HERE, f"c2_{grid}_solve.npz"), eigvals=res["eigvals"],
                        iterations=res["iterations"], converged=res["converged"], timeline=res["timeline"],
                        nev=cfg["nev"], sizeSub=cfg["sizeSub"], seed=cfg["seed"], threads=threads, mu=mu,
                        psi_l1=float(np.sum(np.abs(psi))), psi_max=float(np.max(np.abs(psi))))
    print(grid, "solve", res["iterations"], "iterations", res["converged"], "converged",
          "%.1fs" % (time.time() - t))
    print(res["eigvals"])


def load(name):
    d = np.load(os.path.join(HERE, f"{name}.npz"))
    return {k: d[k] for k in d.files}


if __name__ == "__main__":
    args = sys.argv[1:]
    if args[:1] == ["solve"]:
        # python tests/golden/make_fixtures.py solve c2_64 16 1 [threads]
        solve(args[1], int(args[2]), int(args[3]), int(args[4]) if len(args) > 4 else None)
    elif args[:1] == ["solve_config"]:
        # python tests/golden/make_fixtures.py solve_config 128 psi_128.npz [threads]
        solve_config(int(args[1]), args[2], int(args[3]) if len(args) > 3 else None)
    else:
        for nm in (args or list(PROBLEMS)):
            make(nm)
