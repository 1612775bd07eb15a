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
import os

# OpenBLAS worker threads otherwise spin between BLAS calls and starve the
# OpenMP threads of the reference's CPU FFT (3x slower iterations on 8 cores);
# read when the library loads, so set before numpy / scipy are imported
os.environ.setdefault("OPENBLAS_THREAD_TIMEOUT", "4")
import argparse
import json
import math
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


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cached_solve(grid, mu=None):
    """The full FP64 reference-path solve of this configuration, run once on
    the host (tests/golden/make_fixtures.py solve / solve_config):
    eigenvalues, iterations to tolerance and its per-iteration wall clock.
    None if absent, or if it was made from a psi0 whose mu differs from this
    run's (relative 1e-10)."""
    name = {32: "c1_32", 64: "c2_64", 128: "c2_128"}.get(grid)
    path = os.path.join(ROOT, "tests", "golden", f"{name}_solve.npz") if name else None
    if not path or not os.path.exists(path):
        return None
    d = np.load(path)
    out = {k: d[k] for k in d.files}
    if mu is not None and "mu" in out and abs(float(out["mu"]) - mu) > 1e-10 * abs(mu):
        return None
    return out


def reference_solve_sample(cfg, psi, mu, V, X0, iters, threads):
    """The reference's CPU solve path on the host cores: oracle/_ref, i.e. the
    reference's own src/*.c (bdg_solve -> solver.c -> the iLOBPCG of its
    unvendored LOBPCG dependency, restated; operators through the FFTW-subset
    CPU FFT), set up through its public API, stopped after `iters` whole
    iterations.  Returns the shim's wall-clock timeline: t[0] entry, t[1]
    loop start (Goldstone CG, A X0, Rayleigh-Ritz done), t[2 + i] end of
    iteration i."""
    from oracle import ref as R

    R.set_threads(threads)
    rp = R.build_problem(cfg["N"], cfg["L"], cfg["omegas"], cfg["g"], cfg["gdd"], psi, mu, V=V, Rc=cfg["rc"])
    rp.set_solver_params(cfg["nev"], cfg["sizeSub"], iters, cfg["tol"])
    rp.set_initial_block(X0)
    res = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    rp.close()
    return res["timeline"], res


def reference_anchor_64(threads):
    """A whole reference-path solve timed to tolerance, no projection: the
    64^3 configuration (nev 16, sizeSub 32, true residual <= 1e-8, Goldstone
    chain deflated, X0 ~ N(0, 1) with v = u at seed 1) on the committed
    stationary psi0 of that physics (tests/golden/c2_64.npz, from the
    oracle's ground-state producer).  Returns the line's `anchor_64`."""
    from oracle import ref as R

    f = np.load(os.path.join(ROOT, "tests", "golden", "c2_64.npz"))
    cfg = problem_config(64)
    N, L = [int(v) for v in f["N"]], [float(v) for v in f["L"]]
    R.set_threads(threads)
    t0 = time.perf_counter()
    rp = R.build_problem(N, L, tuple(float(v) for v in f["omegas"]), float(f["g"]), float(f["gdd"]), f["psi"],
                         float(f["mu"]), V=trap(N, L, tuple(float(v) for v in f["omegas"])), Rc=float(f["rc"]))
    u = np.random.default_rng(cfg["seed"]).standard_normal((cfg["sizeSub"], int(np.prod(N))))
    rp.set_solver_params(cfg["nev"], cfg["sizeSub"], 2000, cfg["tol"])
    rp.set_initial_block(np.concatenate([u, u], axis=1))
    res = rp.solve(criterion=R.CONV_TRUE_RESIDUAL, deflate=True)
    rp.close()
    wall = time.perf_counter() - t0
    return {"grid": N, "nev": cfg["nev"], "sizeSub": cfg["sizeSub"], "seconds": wall,
            "iterations": int(res["iterations"]), "converged": int(res["converged"]), "cores": threads,
            "eigenvalues_head": [float(v) for v in res["eigvals"][:4]],
            "what": "one whole reference-path solve to tolerance, timed end to end on the host cores"}


def project_to_tolerance(tl, first, count, cached):
    """Time to tolerance of the reference path from a live sample: the live
    set-up (t[1] - t[0]) plus the cached full solve's loop time scaled by the
    ratio of the live to the cached time of the same iterations
    [first, first + count).  Returns (seconds, live times of the sampled
    iterations, iterations to tolerance)."""
    it_live = np.diff(tl[1:])
    live = it_live[first:first + count]
    if cached is None:
        return None, live, None
    ct = np.asarray(cached["timeline"])
    it_c = np.diff(ct[1:])
    n_tol = int(cached["iterations"])
    ratio = float(np.sum(live) / max(np.sum(it_c[first:first + count]), 1e-12))
    return float(tl[1] - tl[0]) + float(np.sum(it_c[:n_tol])) * ratio, live, n_tol


def reference_inputs(args, cfg):
    """psi0, mu, trap and X0 of the configuration: psi0 from the library's
    GPU ground-state producer (input preparation shared with the GPU arm,
    outside the timed path), or the committed fixture where there is no GPU."""
    V = trap(cfg["N"], cfg["L"], cfg["omegas"])
    psi = mu = None
    try:
        import bdg_lobpcg_b200 as B

        if B.gpu_available():
            psi, mu, _, _, V = ground_state(B, cfg)
    except Exception:
        psi = None
    if psi is None:
        name = {32: "c1_32", 64: "c2_64"}.get(cfg["N"][0])
        if name is None:
            return None
        d = np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"))
        psi, mu = d["psi"], float(d["mu"])
    size = int(np.prod(cfg["N"]))
    u = np.random.default_rng(cfg["seed"]).standard_normal((cfg["sizeSub"], size))
    return psi, mu, V, np.concatenate([u, u], axis=1)


def run_reference(args, cfg):
    """--impl reference: the reference's CPU implementation of the path on the
    host cores, all threads.  One solve of the configuration runs
    warmup + steps whole iterations; step i is iteration warmup + i, timed
    whole (wall clock of the iteration inside the solver).  `value` is the
    time to tolerance projected from those iterations with the cached full
    reference-path solve of the same input (set-up measured live)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    inp = reference_inputs(args, cfg)
    N = cfg["N"]
    if inp is None:
        print(json.dumps({"impl": "reference", "unavailable": f"no psi0 for {N[0]}^3 without a GPU"}))
        return 0
    psi, mu, V, X0 = inp
    threads = os.cpu_count() or 1
    cached = cached_solve(N[0], mu)
    t0 = time.perf_counter()
    tl, res = reference_solve_sample(cfg, psi, mu, V, X0, args.warmup + args.steps, threads)
    wall = time.perf_counter() - t0
    value, live, n_tol = project_to_tolerance(tl, args.warmup, args.steps, cached)
    if value is None:  # no cached full solve: the sampled iterations are the measurement
        value = float(tl[-1] - tl[0])
    sample = (f"one reference-path solve (oracle/_ref: the reference's src/*.c + FFTW-subset CPU FFT + restated "
              f"iLOBPCG, OpenBLAS) of the {N[0]}^3 configuration on {threads} host threads ({cpu_model()}): "
              f"set-up {tl[1] - tl[0]:.1f} s (Goldstone CG, A X0, Rayleigh-Ritz) then {args.warmup} warm-up and "
              f"{args.steps} timed whole iterations; time to tolerance = set-up + the cached full solve's "
              f"{n_tol} iterations scaled by live/cached time of the timed iterations")
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(live)) * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"BdG {N[0]}^3 dipolar trap, nev {cfg['nev']}, sizeSub {cfg['sizeSub']}, "
                                   f"tol 1e-8 (true residual)", "grid": N, "nev": cfg["nev"],
                       "sizeSub": cfg["sizeSub"]},
            "impl": "reference",
            "step_seconds": [float(v) for v in live],
            "setup_seconds": float(tl[1] - tl[0]), "iterations_to_tolerance": n_tol,
            "sample_wall_seconds": wall,
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_anchor:
        try:
            line["anchor_64"] = reference_anchor_64(threads)
        except Exception as e:  # the anchor is a second figure: its failure must not lose the line
            line["anchor_64"] = {"error": f"{type(e).__name__}: {e}"}
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


# ---------------------------------------------------------------------------
# kernel-level workloads (--kernel ops|gram|update): fixed launch sequences for
# ncu captures and CUDA-event timings of single kernels on random blocks
# ---------------------------------------------------------------------------
def model_bytes(op, S, H, e, ec, dipolar=True):
    """Algorithmic bytes per column: e real-space and ec spectrum element size
    (real FP64: 8 and 16; complex FP64: 16 and 16; FP32 halves)."""
    k = 3 * e * S + 4 * ec * H
    m = 3 * e * S + (8 if dipolar else 4) * ec * H
    if op == "LREP":
        return k + m
    if op == "TLREP":
        return 2 * (2 * e * S + 4 * ec * H)
    raise ValueError(op)


def kernel_ops(a):
    """--kernel ops: batched Lrep / T_Lrep applies on random fields of a grid^3
    dipolar context (a fixed launch sequence for ncu), or with --time their
    CUDA-event times per FFT pass family and the bandwidth of the algorithmic
    bytes (three-pass model, model_bytes)."""
    import torch

    import bdg_lobpcg_b200 as B

    N = [a.grid] * 3
    S = a.grid ** 3
    H = S if a.complex else (a.grid // 2 + 1) * a.grid * a.grid
    rng = np.random.default_rng(0)
    dc = B.DeviceContext(3, N, [24.0] * 3, a.complex)
    wf = rng.random(S) + (1j * rng.random(S) if a.complex else 0)
    dc.set_fields(ltK=1 + rng.random(S), ltM=2 + rng.random(S), wf=wf, pK=rng.random(S) + 0.5,
                  pM=rng.random(S) + 0.5, mu=1.0, vdd=rng.standard_normal(H), g_ddi=0.5, dipolar=True)
    if a.complex:
        dt = torch.complex64 if a.prec else torch.complex128
    else:
        dt = torch.float32 if a.prec else torch.float64
    x = torch.randn(a.ncol, 2 * S, dtype=dt, device="cuda")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    if not a.time:
        for op in (B.OP_LREP, B.OP_TLREP):
            for _ in range(1 + a.reps):
                dc.apply_ptr(op, a.prec, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, a.ncol)
        out = torch.zeros(4 * a.ncol * a.ncol * (2 if a.complex else 1), dtype=torch.float64, device="cuda")
        dc.gram_ptr(a.prec, a.complex, S, a.ncol, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, out.data_ptr())
        dc.synchronize()
        print("kernel ops done", a)
        return 0
    stream = torch.cuda.ExternalStream(dc.stream)
    e = (4 if a.prec else 8) * (2 if a.complex else 1)
    ec = 2 * (4 if a.prec else 8)
    for path in a.paths.split(","):
        os.environ["BDG_FFT_PATH"] = path
        for name, op in (("LREP", B.OP_LREP), ("TLREP", B.OP_TLREP)):
            for _ in range(2):
                dc.apply_ptr(op, a.prec, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, a.ncol)
            dc.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(a.reps):
                dc.apply_ptr(op, a.prec, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, a.ncol)
            t1.record(stream)
            t1.synchronize()
            ms = t0.elapsed_time(t1) / a.reps
            gb = model_bytes(name, S, H, e, ec) * a.ncol / 1e9
            print(json.dumps({"path": path, "op": name, "grid": a.grid, "ncol": a.ncol, "prec": a.prec,
                              "complex": a.complex, "ms_per_apply": ms, "ms_per_col": ms / a.ncol,
                              "model_GB": gb, "model_GBps": gb / (ms / 1e3)}))
    return 0


def _time(fn, stream, reps):
    import torch

    fn()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(reps):
        fn()
    t1.record(stream)
    t1.synchronize()
    return t0.elapsed_time(t1) / reps


def kernel_gram(a):
    """--kernel gram: bdgd_gram (Guu, Gvv, Guv, Ga of a --k column block on
    2 grid^3 rows) against cuBLAS FP64 on the same contraction and on 8192^3."""
    import torch

    import bdg_lobpcg_b200 as B

    k, S = a.k, a.grid ** 3
    n = 2 * S
    if a.complex:
        dt = torch.complex64 if a.prec else torch.complex128
    else:
        dt = torch.float32 if a.prec else torch.float64
    dc = B.DeviceContext(3, [a.grid] * 3, [24.0] * 3, a.complex)
    X = torch.randn(k, n, dtype=dt, device="cuda")
    AX = torch.randn(k, n, dtype=dt, device="cuda")
    out = torch.zeros(4 * k * k * (2 if a.complex else 1), dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(dc.stream)

    def lib():
        dc.gram_ptr(a.prec, a.complex, S, k, X.data_ptr(), n, AX.data_ptr(), n, out.data_ptr())

    ms = _time(lib, stream, a.reps)
    tiles = (k + 63) // 64
    symfrac = tiles * (tiles + 1) / 2 / (tiles * tiles)
    cf = 4.0 if a.complex else 1.0  # real flops per complex multiply-add pair
    flops_exec = cf * (2.0 * S * k * k * (2 * symfrac + 1) + 2.0 * n * k * k)
    flops_min = cf * (2.0 * S * k * k * 2 + 2.0 * n * k * k)  # Guu, Gvv half each + Guv + Ga
    print(json.dumps({"what": "bdgd_gram", "k": k, "rows": n, "prec": a.prec, "complex": a.complex, "ms": ms,
                      "tflops_executed": flops_exec / ms / 1e9, "tflops_useful": flops_min / ms / 1e9}))
    if a.complex:
        return 0
    Xd, AXd = X.double(), AX.double()
    cur = torch.cuda.current_stream()
    ms2 = _time(lambda: (torch.mm(Xd, Xd.t()), torch.mm(Xd, AXd.t())), cur, a.reps)
    print(json.dumps({"what": "cublas_fp64_same_contraction", "k": k, "rows": n, "ms": ms2,
                      "tflops": 2 * 2.0 * n * k * k / ms2 / 1e9}))
    M = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    ms3 = _time(lambda: torch.mm(M, M), cur, a.reps)
    print(json.dumps({"what": "cublas_fp64_square_8192", "ms": ms3, "tflops": 2.0 * 8192 ** 3 / ms3 / 1e9}))
    return 0


def kernel_update(a):
    """--kernel update: the basis update of one iteration (bdgd_block_update,
    four outputs) and the projection shape against cuBLAS FP64."""
    import torch

    import bdg_lobpcg_b200 as B

    m, n = a.k, 2 * a.grid ** 3
    dc = B.DeviceContext(3, [a.grid] * 3, [24.0] * 3, False)
    blk = {nm: torch.randn(m, n, dtype=torch.float64, device="cuda") for nm in ("X", "P", "W", "AX", "AP", "AW")}
    out = {nm: torch.empty(m, n, dtype=torch.float64, device="cuda") for nm in ("XN", "AXN", "PN", "APN")}
    Cx = torch.randn(m, 3 * m, dtype=torch.float64, device="cuda")  # (3m x m) column-major
    Cp = torch.randn(m, 2 * m, dtype=torch.float64, device="cuda")  # (2m x m) column-major
    stream = torch.cuda.ExternalStream(dc.stream)
    e8 = 8

    def terms(names, Cm, k):
        return [(blk[nm].data_ptr(), m, Cm.data_ptr() + i * m * e8, k) for i, nm in enumerate(names)]

    outs = [(out["XN"].data_ptr(), m, 1.0, 0.0, terms(("X", "P", "W"), Cx, 3 * m)),
            (out["AXN"].data_ptr(), m, 1.0, 0.0, terms(("AX", "AP", "AW"), Cx, 3 * m)),
            (out["PN"].data_ptr(), m, 1.0, 0.0, terms(("P", "W"), Cp, 2 * m)),
            (out["APN"].data_ptr(), m, 1.0, 0.0, terms(("AP", "AW"), Cp, 2 * m))]

    def lib():
        rc = dc.block_update(0, False, n, n, outs)
        if rc:
            raise RuntimeError(f"bdgd_block_update: {rc}")

    flops = 2.0 * n * m * (3 * m * 2 + 2 * m * 2)
    ms = _time(lib, stream, a.reps)
    print(json.dumps({"what": "bdgd_block_update", "m": m, "rows": n, "ms": ms, "tflops": flops / ms / 1e9}))
    # reference: the same products as cuBLAS GEMMs (rows of the torch tensors are columns of the blocks)
    Sx = torch.cat([blk["X"], blk["P"], blk["W"]])
    Sa = torch.cat([blk["AX"], blk["AP"], blk["AW"]])
    cur = torch.cuda.current_stream()

    def blas():
        torch.mm(Cx, Sx, out=out["XN"])
        torch.mm(Cx, Sa, out=out["AXN"])
        torch.mm(Cp, Sx[m:], out=out["PN"])
        torch.mm(Cp, Sa[m:], out=out["APN"])

    ms2 = _time(blas, cur, a.reps)
    print(json.dumps({"what": "cublas_fp64_same_products", "m": m, "rows": n, "ms": ms2, "tflops": flops / ms2 / 1e9}))
    # projection shape: P -= X Cs, AP -= AX Cs (k = m, beta = 1), two outputs
    Cs = torch.randn(m, m, dtype=torch.float64, device="cuda")
    pouts = [(out["PN"].data_ptr(), m, -1.0, 1.0, [(blk["X"].data_ptr(), m, Cs.data_ptr(), m)]),
             (out["APN"].data_ptr(), m, -1.0, 1.0, [(blk["AX"].data_ptr(), m, Cs.data_ptr(), m)])]

    def libp():
        rc = dc.block_update(0, False, n, n, pouts)
        if rc:
            raise RuntimeError(f"bdgd_block_update: {rc}")

    pflops = 2.0 * n * m * m * 2
    ms = _time(libp, stream, a.reps)
    print(json.dumps({"what": "bdgd_block_update_projection", "m": m, "rows": n, "ms": ms,
                      "tflops": pflops / ms / 1e9}))

    def blasp():
        out["PN"].addmm_(Cs, blk["X"], alpha=-1.0)
        out["APN"].addmm_(Cs, blk["AX"], alpha=-1.0)

    ms2 = _time(blasp, cur, a.reps)
    print(json.dumps({"what": "cublas_fp64_projection", "m": m, "rows": n, "ms": ms2, "tflops": pflops / ms2 / 1e9}))
    # agreement of the two on the last outputs
    lib()
    torch.cuda.synchronize()
    ref = torch.mm(Cp, Sa[m:])
    err = float((out["APN"] - ref).abs().max() / ref.abs().max())
    print(json.dumps({"what": "max_rel_diff_APN", "value": err}))
    return 0



def kernel_main(argv):
    ap = argparse.ArgumentParser(prog="bench.py --kernel")
    ap.add_argument("--kernel", required=True, choices=["ops", "gram", "update"])
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--ncol", type=int, default=8)
    ap.add_argument("--k", type=int, default=192, help="block columns (gram) / columns per block (update)")
    ap.add_argument("--prec", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--complex", action="store_true")
    ap.add_argument("--time", action="store_true")
    ap.add_argument("--paths", default="reg,ct")
    a = ap.parse_args(argv)
    return {"ops": kernel_ops, "gram": kernel_gram, "update": kernel_update}[a.kernel](a)


def c3_config():
    """The complex (_z) configuration: 128^3 in [-12, 12)^3, lambda 1, g 1500,
    eps_dd 0.4, R_c 8, nev 48 (sizeSub 96), tol 1e-8 on the true residual,
    complex N(0, 1) initial block (v = u) at seed 2."""
    g = 1500.0
    return dict(N=[128] * 3, L=[24.0] * 3, omegas=(1.0, 1.0, 1.0), g=g, gdd=0.4 * g, eps_dd=0.4, lam=1.0, rc=8.0,
                nev=48, sizeSub=96, tol=1e-8, seed=2)


def run_c3(args):
    """--config c3: the complex path at 128^3, complex128 and complex64 with
    FP64 refinement, on psi0 = e^{0.7 i} psi_real (a genuinely complex
    condensate; the fixed-winding vortex of this physics makes K = H - mu
    indefinite, outside the definite-pencil iLOBPCG), Goldstone chain
    deflated.  Prints one JSON line with both forms."""
    import bdg_lobpcg_b200 as B
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if not B.gpu_available():
        raise RuntimeError("bench needs a CUDA device")
    cfg = c3_config()
    psi, mu, itp_steps, stationarity, V = ground_state(B, cfg)
    psi_z = psi * np.exp(0.7j)
    size = int(np.prod(cfg["N"]))
    rng = np.random.default_rng(cfg["seed"])
    u = rng.standard_normal((cfg["sizeSub"], size)) + 1j * rng.standard_normal((cfg["sizeSub"], size))
    X0 = np.concatenate([u, u], axis=1)
    forms = {}
    for prec in ("f64", "mixed"):
        p = B.Problem(3, cfg["N"], cfg["L"], complex_psi0=True)
        p.set_system()
        p.set_trap(V)
        p.set_wavefunction(psi_z)
        g = cfg["g"]
        p.set_local_interactions(lambda n: g * n, lambda n: g * n)
        p.set_dipolar(cfg["gdd"], [0.0, 0.0, 1.0], cfg["rc"])
        p.set_mu(mu)
        p.set_solver_params(cfg["nev"], cfg["sizeSub"], 2000, cfg["tol"])
        p.set_convergence(B.CONV_TRUE_RESIDUAL)
        p.set_goldstone_deflation(True)
        p.set_precision(B.PREC_MIXED if prec == "mixed" else B.PREC_F64)
        p.set_initial_block(X0)
        for _ in range(args.warmup):
            if p.solve():
                raise RuntimeError("bdg_solve (complex) failed")
        dev, e2e = [], []
        for _ in range(args.steps):
            t = time.perf_counter()
            if p.solve():
                raise RuntimeError("bdg_solve (complex) failed")
            e2e.append(time.perf_counter() - t)
            dev.append(p.stats()["seconds_device"])
        st = p.stats()
        forms[prec] = {"value": float(np.mean(dev)), "e2e": float(np.mean(e2e)), "unit": "s",
                       "iterations": st["iterations"], "refine_iterations": st["refine_iterations"],
                       "converged": p.converged(), "max_true_residual": st["max_true_residual"],
                       "eigenvalues": [float(v) for v in p.eigenvalues()],
                       "stage_ms": {k: st[k] for k in ("ms_apply_A", "ms_apply_T", "ms_residual", "ms_gram",
                                                        "ms_small_dense", "ms_update")}}
        p.close()
    ef = np.asarray(forms["f64"]["eigenvalues"])
    em = np.asarray(forms["mixed"]["eigenvalues"])
    line = {"metric": "time to res<=1e-8, 48 BdG modes @128^3, complex path", "value": forms["f64"]["value"],
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": "complex BdG 128^3 dipolar trap (eps_dd 0.4, lambda 1, g 1500), psi0 = "
                                   "e^{0.7i} psi_real, nev 48, sizeSub 96, tol 1e-8 true residual, deflated",
                       "grid": cfg["N"], "nev": cfg["nev"], "sizeSub": cfg["sizeSub"]},
            "ground_state": {"mu": mu, "itp_steps": itp_steps, "stationarity": stationarity},
            "complex128": forms["f64"], "complex64_fp64": forms["mixed"],
            "eig_rel_err_mixed_vs_c128": float(np.max(np.abs(em - ef) / np.abs(ef)))}
    print(json.dumps(line))
    return 0


def main():
    if "--kernel" in sys.argv[1:]:
        return kernel_main(sys.argv[1:])
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--precision", default="f64", choices=["f64", "mixed"])
    ap.add_argument("--config", default="c2", choices=["c2", "c3"],
                    help="c2: the 128^3 real headline; c3: the complex path (own JSON line)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-baseline-iters", type=int, default=1,
                    help="whole reference-path iterations timed for cpu_baseline")
    ap.add_argument("--no-anchor", action="store_true",
                    help="--impl reference: skip the whole 64^3 reference-path solve timed beside the sample")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the mixed-precision variant measured beside the FP64 headline")
    args = ap.parse_args()
    cfg = problem_config(args.grid)
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.config == "c3":
        return run_c3(args)

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
    variants = {}
    if not args.no_variants and args.precision == "f64":
        # the mixed FP32/FP64 form of the same solve (same psi0, X0), timed the same way
        pm, _ = build(B, cfg, psi, mu, V, "mixed")
        for _ in range(args.warmup):
            pm.solve()
        mt, me = [], []
        for _ in range(args.steps):
            t = time.perf_counter()
            rc = pm.solve()
            me.append(time.perf_counter() - t)
            if rc:
                raise RuntimeError(f"bdg_solve (mixed) failed ({rc})")
            mt.append(pm.stats()["seconds_device"])
        sm = pm.stats()
        em = pm.eigenvalues()
        ef = p.eigenvalues()
        variants["mixed"] = {
            "value": float(np.mean(mt)), "e2e": float(np.mean(me)), "unit": "s",
            "iterations": sm["iterations"], "refine_iterations": sm["refine_iterations"],
            "max_true_residual": sm["max_true_residual"], "converged": pm.converged(),
            "eig_rel_err_vs_f64_gpu": float(np.max(np.abs(em - ef) / np.abs(ef))),
            "eigenvalues": [float(v) for v in em]}
        pm.close()
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
    cached = cached_solve(cfg["N"][0], mu)
    ce = None
    if cached is not None:
        # per-eigenvalue relative error against the FP64 CPU oracle solve of the same input
        ce = np.asarray(cached["eigvals"])[: cfg["nev"]]
        line["eig_rel_err_vs_cpu_oracle"] = float(np.max(np.abs(ev[: cfg["nev"]] - ce) / np.abs(ce)))
    if variants:
        for v in variants.values():
            e = np.asarray(v.pop("eigenvalues"))[: cfg["nev"]]
            if ce is not None:
                v["eig_rel_err_vs_cpu_oracle"] = float(np.max(np.abs(e - ce) / np.abs(ce)))
        line["variants"] = variants
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        k = max(1, args.cpu_baseline_iters)
        tl, _ = reference_solve_sample(cfg, psi, mu, V, X0, k, threads)
        cval, live, n_tol = project_to_tolerance(tl, 0, k, cached)
        line["cpu_baseline"] = {
            "value": cval if cval is not None else float(tl[-1] - tl[0]), "unit": "s", "cores": threads,
            "kind": "reference",
            "sample": f"reference-path solve (oracle/_ref) of the same input on {threads} host threads "
                      f"({cpu_model()}): set-up {tl[1] - tl[0]:.1f} s + {k} whole iteration(s) "
                      f"({', '.join(f'{v:.1f}' for v in live)} s), projected to the {n_tol} iterations of the "
                      f"cached full reference-path solve"}
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
