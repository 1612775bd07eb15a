#!/usr/bin/env python
"""Benchmark of the BdG operator-and-solver path on B200.

Metric: time until the 32 lowest BdG modes of the 128^3 dipolar trap reach a
true residual ||K M v - w^2 v|| / ||v|| <= 1e-8 (seconds, lower is better).
Workload (the 128^3 configuration of the benchmark description): box
[-12, 12)^3, trap (1, 1, lambda = 2), g = 1000, eps_dd = 0.7 (g_dd = 700),
dipoles along z, cutoff radius 8; psi0 = stationary ground state (GPU
split-step imaginary time, dt = 1e-3 until |d mu| < 1e-12, then Newton
polish); nev 32, sizeSub 64, Goldstone chain deflated, initial block
X0 ~ N(0,1) at seed 1 with v = u (B-positive).  Synthetic data (no external
inputs exist for this problem).

One step = one full solve.  `value` = device time of the iteration loop
(inputs resident in HBM, CUDA events inside the library); `e2e` = wall time
of the public bdg_solve call, which uploads the host initial block, iterates
and downloads eigenvalues and modes.  Inputs are far larger than L2 (the
iteration streams ~30 GB of blocks), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--grid 128] [--precision f64|mixed]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from bdg_lobpcg_b200 import problems  # noqa: E402

METRIC = "time to res<=1e-8, 32 BdG modes @128^3"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# DRAM read + write bytes per column of a real Lrep apply, summed over the
# five pass kernels of one 8-column launch captured with ncu (128^3 FP64)
LREP_DRAM_BYTES_PER_COLUMN = {(128, "f64"): 480.4e6}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def problem_config(grid):
    return problems.config(grid)


grid_coords, trap = problems.grid_coords, problems.trap


def ground_state(B, cfg):
    return problems.ground_state(B, cfg)


def build(B, cfg, psi, mu, V, precision):
    return problems.build(B, cfg, psi, mu, V, precision)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([v.strip() for v in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(s[1]) for s in self.samples if len(s) > 8 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 8 and s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            if len(s) > 8:
                for nm, v in zip(names, s[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def cpu_sample(cfg, psi, mu, V, X0, n_cols=2):
    """Oracle port (numpy/scipy, all host threads): time the per-iteration work
    of the same solve on a bounded sample -- n_cols columns of A and T applies
    plus the Gram/Rayleigh-Ritz and update dense work at the full block size
    -- and return seconds per iteration."""
    from oracle import bdg_oracle as O

    oc = O.build_problem(cfg["N"], cfg["L"], cfg["omegas"], cfg["g"], cfg["gdd"], psi, mu, Rc=cfg["rc"])
    m = cfg["sizeSub"]
    Xs = X0[:n_cols]
    t = time.perf_counter()
    AX = O.matmulLrep(oc, Xs)
    t_a = (time.perf_counter() - t) / n_cols
    t = time.perf_counter()
    O.precondLrep(oc, Xs)
    t_t = (time.perf_counter() - t) / n_cols
    # dense: Gram blocks of a 3m-column basis against itself and its A-image,
    # measured on a 3m x (rows) slice and scaled to the full row count
    rows = min(oc.size * 2, 1 << 19)
    S3 = np.random.default_rng(0).standard_normal((3 * m, rows))
    t = time.perf_counter()
    _ = S3 @ S3.T
    _ = S3 @ S3.T
    _ = S3[:, : rows // 2] @ S3[:, rows // 2:].T
    t_g = (time.perf_counter() - t) * (2 * oc.size / rows)
    t = time.perf_counter()
    _ = S3.T @ np.ones((3 * m, m))
    t_u = (time.perf_counter() - t) * 4 * (2 * oc.size / rows)
    per_iter = m * (t_a + t_t) + t_g + t_u
    return per_iter, {"A_per_col_s": t_a, "T_per_col_s": t_t, "gram_s": t_g, "update_s": t_u}


def run_reference(args, cfg):
    """The reference's CPU path: the reference's FFTW/LOBPCG dependencies are
    absent here, so its algorithm runs as the oracle port (numpy/scipy with
    all host threads).  Each step = a bounded sample of one iteration; the
    reported value is the estimated time to tolerance (per-iteration time x
    the iteration count the same solve needs)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import bdg_oracle as O

    N, L = cfg["N"], cfg["L"]
    # psi0: the fixture for 32^3, else an oracle ITP would take hours at
    # 128^3 on the host, so the CPU sample uses a Thomas-Fermi profile of the
    # same trap (the per-iteration work does not depend on psi0).
    V = trap(N, L, cfg["omegas"])
    if N[0] == 32:
        sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
        import make_fixtures as FX

        fx = FX.load("c1_32")
        psi, mu = fx["psi"], float(fx["mu"])
    else:
        mu = 20.0
        psi = np.sqrt(np.clip((mu - V) / cfg["g"], 0, None))
        psi /= math.sqrt(np.sum(psi ** 2) * np.prod([l / n for l, n in zip(L, N)]))
    size = int(np.prod(N))
    rng = np.random.default_rng(cfg["seed"])
    u = rng.standard_normal((4, size))
    X0 = np.concatenate([u, u], axis=1)
    iters_needed = args.ref_iters
    times = []
    for i in range(args.warmup + args.steps):
        per_iter, parts = cpu_sample(cfg, psi, mu, V, X0)
        if i >= args.warmup:
            times.append(per_iter * iters_needed)
    value = float(np.mean(times))
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"BdG {N[0]}^3 dipolar trap, nev {cfg['nev']}, sizeSub {cfg['sizeSub']}, "
                                   f"tol 1e-8 (true residual)", "grid": N, "nev": cfg["nev"]},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"one iLOBPCG iteration of the oracle port (numpy/scipy FFT, "
                                       f"{os.cpu_count()} threads) at {N[0]}^3, sizeSub {cfg['sizeSub']}, "
                                       f"x {iters_needed} iterations; per-iteration parts {parts}"},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def max_over_ranks(values, dist, device):
    """Per-rank timings reduced to their maximum over all ranks (every rank
    calls this, in the same order; `device` is "cuda" under NCCL and "cpu"
    under gloo)."""
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def gram_roofline(B, torch, cfg, reps=5):
    """The dominant kernel: the FP64 Gram contraction (k_gram_sk, DMMA) at the
    solve's shapes (k = 3 sizeSub columns of S and AS on 2 N^3 rows: Guu, Gvv,
    Guv, Ga), timed with CUDA events on the library's stream, against cuBLAS
    FP64 GEMM 8192^3 measured in the same process (the FP64 tensor-core
    reference; the measured-peaks file holds no FP64 figure)."""
    size = int(np.prod(cfg["N"]))
    n, k = 2 * size, 3 * cfg["sizeSub"]
    dc = B.DeviceContext(3, cfg["N"], cfg["L"], False)
    gen = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn(k, n, dtype=torch.float64, device="cuda", generator=gen)
    AX = torch.randn(k, n, dtype=torch.float64, device="cuda", generator=gen)
    out = torch.zeros(4 * k * k, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(dc.stream)

    def timed(fn, st):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    ms = timed(lambda: dc.gram_ptr(0, False, size, k, X.data_ptr(), n, AX.data_ptr(), n, out.data_ptr()), stream)
    tiles = (k + 63) // 64
    symfrac = tiles * (tiles + 1) / 2 / (tiles * tiles)
    flops = 2.0 * size * k * k * (2 * symfrac + 1) + 2.0 * n * k * k  # tiles computed
    del X, AX
    M = torch.randn(8192, 8192, dtype=torch.float64, device="cuda", generator=gen)
    cur = torch.cuda.current_stream()
    ms_ref = timed(lambda: torch.mm(M, M), cur)
    ref = 2.0 * 8192 ** 3 / ms_ref / 1e9
    dc.close()
    achieved = flops / ms / 1e9
    return {"bound": "tensor (FP64 DMMA)", "kernel": f"k_gram_sk: Gram of S, AS (k = {k}, rows = {n})",
            "achieved": achieved, "peak": ref, "unit": "TFLOP/s", "frac": achieved / ref,
            "peak_kind": "cuBLAS FP64 GEMM 8192^3 measured in this run", "ms_per_launch": ms,
            "flops_per_launch": flops, "traffic": None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--precision", default="f64", choices=["f64", "mixed"])
    ap.add_argument("--ref-iters", type=int, default=80,
                    help="iterations used to scale the reference per-iteration sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    cfg = problem_config(args.grid)
    if args.impl == "reference":
        return run_reference(args, cfg)

    import bdg_lobpcg_b200 as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    if not B.gpu_available():
        raise RuntimeError("bench needs a CUDA device")
    t_setup = time.perf_counter()
    psi, mu, itp_steps, stationarity, V = ground_state(B, cfg)
    t_gs = time.perf_counter() - t_setup
    p, X0 = build(B, cfg, psi, mu, V, args.precision)
    L = B.lib()
    # warm-up solves (untimed)
    for _ in range(args.warmup):
        rc = p.solve()
        if rc:
            raise RuntimeError(f"bdg_solve failed ({rc})")
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = L.bdgd_launch_count()
    dev_times, e2e_times, stats = [], [], []
    for _ in range(args.steps):
        t = time.perf_counter()
        rc = p.solve()
        e2e_times.append(time.perf_counter() - t)
        if rc:
            raise RuntimeError(f"bdg_solve failed ({rc})")
        st = p.stats()
        dev_times.append(st["seconds_device"])
        stats.append(st)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    launches = L.bdgd_launch_count() - launches0
    ck = clocks.stop()
    value = float(np.mean(dev_times))
    e2e = float(np.mean(e2e_times))
    if pg:
        value, e2e = max_over_ranks([value, e2e], pg, "cuda")
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return 0
    st = stats[-1]
    ev = p.eigenvalues()
    size = int(np.prod(cfg["N"]))
    peaks, peak_kind = load_peaks()
    # roofline of the batched Lrep apply (5 FFT pass kernels per launch):
    # algorithmic bytes per column from the 3-pass FFT-round-trip model
    e = 8 if args.precision == "f64" else 4
    H = (cfg["N"][0] // 2 + 1) * cfg["N"][1] * cfg["N"][2]
    lrep_bytes = 6 * e * size + 12 * 2 * e * H
    t_bytes = 2 * (2 * e * size + 4 * 2 * e * H)
    a_gbs = lrep_bytes * st["cols_apply_A"] / (st["ms_apply_A"] * 1e-3) / 1e9 if st["ms_apply_A"] else None
    t_gbs = t_bytes * st["cols_apply_T"] / (st["ms_apply_T"] * 1e-3) / 1e9 if st["ms_apply_T"] else None
    peak = peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    n = 2 * size
    h2d = n * cfg["sizeSub"] * 8 + size * 8 * 4  # initial block + fields
    d2h = 2 * size * cfg["nev"] * 8 + cfg["nev"] * 8  # the nev modes (u and v halves) + eigenvalues
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "f64" else "f32+f64",
        "data": "synthetic",
        "config": {"workload": f"BdG {cfg['N'][0]}^3 dipolar trap (eps_dd {cfg['gdd'] / cfg['g']:.1f}, lambda 2, "
                               f"g 1000), nev {cfg['nev']}, sizeSub {cfg['sizeSub']}, tol 1e-8 true residual",
                   "grid": cfg["N"], "nev": cfg["nev"], "sizeSub": cfg["sizeSub"], "precision": args.precision,
                   "parallelism": "replicas" if world > 1 else "single", "l2": "inputs >> L2 (no flush)"},
        "iterations": st["iterations"], "refine_iterations": st["refine_iterations"],
        "max_true_residual": st["max_true_residual"], "converged": p.converged(),
        "eigenvalues_head": [float(v) for v in ev[:6]],
        "stage_ms": {k: st[k] for k in ("ms_apply_A", "ms_apply_T", "ms_residual", "ms_gram", "ms_small_dense",
                                         "ms_update")},
        "e2e_split_s": {"setup": st["seconds_setup"], "loop_device": st["seconds_device"],
                        "output": st["seconds_output"], "bdg_solve_wall": st["seconds_total"]},
        "ground_state": {"seconds": t_gs, "itp_steps": itp_steps, "mu": mu, "stationarity": stationarity},
        "roofline": {"bound": "hbm", "kernel": "batched Lrep apply (5 FFT pass kernels)",
                     "achieved": a_gbs, "peak": peak, "unit": "GB/s",
                     "frac": (a_gbs / peak) if a_gbs else None, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_column": lrep_bytes,
                     "traffic": LREP_DRAM_BYTES_PER_COLUMN.get((cfg["N"][0], args.precision)),
                     "traffic_basis": "DRAM bytes per column (ncu, 8-column launches of the five pass kernels)",
                     "precond_achieved": t_gbs},
        "roofline_gram": gram_roofline(B, torch, cfg) if args.precision == "f64" else None,
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": ck,
    }
    if not args.no_cpu_baseline:
        per_iter, parts = cpu_sample(cfg, psi, mu, V, X0)
        line["cpu_baseline"] = {"value": per_iter * st["iterations"], "unit": "s", "cores": os.cpu_count(),
                                "kind": "port",
                                "sample": f"oracle port per-iteration work at {cfg['N'][0]}^3 (2 columns of A and "
                                          f"T scaled to {cfg['sizeSub']}, Gram/update dense work scaled from a row "
                                          f"slice) x {st['iterations']} iterations; parts {parts}"}
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
