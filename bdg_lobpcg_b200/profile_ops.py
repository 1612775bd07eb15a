"""Batched operator applies for profiling (ncu) and timing.

    python -m bdg_lobpcg_b200.profile_ops [--grid 128] [--ncol 8] [--prec 0|1] [--reps 3]
                                          [--complex] [--time] [--paths reg,ct]
    python -m bdg_lobpcg_b200.profile_ops --gram 192 [--grid 128] [--prec 0|1] [--reps 5]
    python -m bdg_lobpcg_b200.profile_ops --update 64 [--grid 128] [--reps 5]

Random fields and columns on a grid^3 dipolar context.  Without --time it
applies LREP and TLREP `reps` times each (after one warm-up apply), then one
Gram of the block: a fixed launch sequence for ncu.  With --time it times
`reps` applies of each operator per FFT pass family with CUDA events on the
library's stream and prints one JSON line per (path, operator) with the
milliseconds per apply and the bandwidth of the algorithmic bytes (the
three-pass FFT round-trip model: per column K = 3e*S + 4*ec*H,
M = 3e*S + 8*ec*H with the dipolar exchange, T_Lrep = 2*(2e*S + 4*ec*H),
e the real-space and ec the spectrum element size, H the spectrum points
per field).

With --gram K it times bdgd_gram (Guu, Gvv, Guv and Ga of a K-column block
on 2*grid^3 rows) and, for reference, cuBLAS FP64 through torch on the same
contraction (S S^T and S AS^T of the K x n blocks) and on a square 8192^3
FP64 GEMM, and prints the FLOP rates.  The library counts a symmetric block
at tile granularity (64 x 64 tiles on and above the diagonal).

With --update M it times the iLOBPCG basis update of one iteration on
2*grid^3 rows with M columns per block: X' = [X P W] C_x and
P' = [P W] C_p with their A-images (four outputs, one launch of
bdgd_block_update), against the same products as four cuBLAS FP64 GEMMs
through torch, and prints the FLOP rates.
"""
import argparse
import json
import os
import sys

import numpy as np


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--ncol", type=int, default=8)
    ap.add_argument("--prec", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--complex", action="store_true")
    ap.add_argument("--time", action="store_true")
    ap.add_argument("--paths", default="reg,ct")
    ap.add_argument("--gram", type=int, default=0)
    ap.add_argument("--update", type=int, default=0)
    a = ap.parse_args()
    import torch

    if a.gram:
        return gram_main(a)
    if a.update:
        return update_main(a)

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
        print("profile_ops done", a)
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


def gram_main(a):
    import torch

    import bdg_lobpcg_b200 as B

    k, S = a.gram, a.grid ** 3
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


def update_main(a):
    import torch

    import bdg_lobpcg_b200 as B

    m, n = a.update, 2 * a.grid ** 3
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


if __name__ == "__main__":
    sys.exit(main())
