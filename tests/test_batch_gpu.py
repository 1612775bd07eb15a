"""Batched solves, CUDA-graph replay and the FFT autotuner (GPU).

* bdg_solve_batch on three problems of different grids gives the same
  eigenvalues (1e-12 relative) as solving them one at a time;
* operator applies replayed from CUDA graphs give the same result as direct
  launches (bit-identical: same kernels, same inputs), and a field setter
  invalidates a recorded graph;
* the autotuner times both FFT pass families and keeps the faster.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


def test_batch_matches_sequential(bdg):
    from bdg_lobpcg_b200 import problems

    cfgs = [problems.config(32, nev=4), problems.config(32, eps_dd=0.3, lam=1.5, nev=4, seed=5),
            problems.config(16, box=12.0, nev=4, seed=6)]
    states = [problems.ground_state(bdg, c) for c in cfgs]

    def build():
        return [problems.build(bdg, c, *s[:2], s[4])[0] for c, s in zip(cfgs, states)]

    seq = []
    for p in build():
        assert p.solve() == 0
        seq.append(p.eigenvalues().copy())
        p.close()
    probs = build()
    rcs, secs = bdg.solve_batch(probs, concurrency=3, graphs=True)
    assert rcs == [0, 0, 0] and np.all(secs > 0)
    for p, e in zip(probs, seq):
        assert np.max(np.abs(p.eigenvalues() - e) / np.abs(e)) < 1e-12
        assert p.stats()["max_true_residual"] <= 1e-8
        p.close()


def _ctx(bdg, rng, N=(32, 32, 32)):
    S = int(np.prod(N))
    H = (N[0] // 2 + 1) * S // N[0]
    dc = bdg.DeviceContext(3, list(N), [12.0] * 3, False)
    dc.set_fields(ltK=1 + rng.random(S), ltM=2 + rng.random(S), wf=rng.standard_normal(S), pK=0.5 + rng.random(S),
                  pM=0.5 + rng.random(S), mu=0.7, vdd=rng.standard_normal(H), g_ddi=0.4, dipolar=True)
    return dc, S


def test_graph_replay_matches_direct(bdg, monkeypatch):
    torch = _torch()
    monkeypatch.setenv("BDG_FFT_PATH", "reg")
    rng = np.random.default_rng(2)
    dc, S = _ctx(bdg, rng)
    x = torch.randn(6, 2 * S, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    torch.cuda.synchronize()
    dc.apply_ptr(bdg.OP_LREP, 0, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, 6)
    dc.synchronize()
    ref = y.clone()
    dc.set_graphs(True)
    for _ in range(4):  # direct, capture + launch, replay, replay
        y.zero_()
        torch.cuda.synchronize()
        dc.apply_ptr(bdg.OP_LREP, 0, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, 6)
        dc.synchronize()
        assert torch.equal(y, ref)
    # a setter changes mu: the recorded graph must not be replayed
    dc.set_fields(ltK=1 + rng.random(S), ltM=2 + rng.random(S), wf=rng.standard_normal(S), pK=0.5 + rng.random(S),
                  pM=0.5 + rng.random(S), mu=0.9, vdd=rng.standard_normal((S // 32) * 17), g_ddi=0.4, dipolar=True)
    dc.set_graphs(False)
    dc.apply_ptr(bdg.OP_TLREP, 0, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, 6)
    dc.synchronize()
    ref2 = y.clone()
    dc.set_graphs(True)
    for _ in range(3):
        y.zero_()
        torch.cuda.synchronize()
        dc.apply_ptr(bdg.OP_TLREP, 0, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, 6)
        dc.synchronize()
        assert torch.equal(y, ref2)


def test_autotuner_picks_faster_family(bdg, monkeypatch):
    torch = _torch()
    monkeypatch.delenv("BDG_FFT_PATH", raising=False)
    monkeypatch.delenv("BDG_GENERIC_FFT", raising=False)
    rng = np.random.default_rng(3)
    dc, S = _ctx(bdg, rng)
    x = torch.randn(8, 2 * S, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    torch.cuda.synchronize()
    assert dc.fft_tuning(bdg.OP_LREP, 0)[0] == 0
    dc.apply_ptr(bdg.OP_LREP, 0, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, 8)
    dc.synchronize()
    path, ms = dc.fft_tuning(bdg.OP_LREP, 0)
    assert path in (1, 2) and ms[0] > 0 and ms[1] > 0
    assert ms[path - 1] <= ms[2 - path]
    # the tuned apply gives the operator (same as the fixed register family)
    tuned = y.clone()
    monkeypatch.setenv("BDG_FFT_PATH", "reg")
    dc.apply_ptr(bdg.OP_LREP, 0, x.data_ptr(), 2 * S, y.data_ptr(), 2 * S, 8)
    dc.synchronize()
    assert float((tuned - y).abs().max() / y.abs().max()) < 1e-12
