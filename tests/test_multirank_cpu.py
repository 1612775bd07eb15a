"""Multi-rank host logic on the CPU: two gloo ranks, no GPU.

One BdG problem runs on one GPU; several GPUs run independent work (replicas
of the bench solve, or shards of the batched sweep), so the only cross-rank
steps are host-side:
* the bench's timing is the maximum over ranks (`bench.max_over_ranks`);
* the sweep shards its problems round robin and rank 0 gathers the
  per-problem records (`sweep.shard`, `sweep.merge_shards`, gather_object);
* the reference arm does its work on rank 0 only and the other ranks exit 0
  without output.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from bdg_lobpcg_b200 import sweep

        vals = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5], dist, "cpu")
        n = 7
        mine = sweep.shard(n, rank, world)
        recs = [(i, {"i": i, "rank": rank}) for i in mine]
        out = [None] * world if rank == 0 else None
        dist.gather_object(recs, out, dst=0)
        merged = sweep.merge_shards(n, out) if rank == 0 else None
        q.put((rank, vals, mine, merged))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_sweep_gather():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, vals, mine, merged = q.get(timeout=120)
        res[rank] = (vals, mine, merged)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert res[r][0] == [2.0, 10.0, 0.5]  # max over ranks, element by element
    assert res[0][1] == [0, 2, 4, 6] and res[1][1] == [1, 3, 5]
    merged = res[0][2]
    assert [m["i"] for m in merged] == list(range(7))
    assert [m["rank"] for m in merged] == [i % 2 for i in range(7)]
    assert res[1][2] is None


def test_shard_and_merge_edge_cases():
    from bdg_lobpcg_b200 import sweep

    assert sweep.shard(3, 2, 4) == [2] and sweep.shard(3, 3, 4) == []  # more ranks than problems
    assert sweep.merge_shards(0, [[], []]) == []
    with pytest.raises(ValueError):
        sweep.merge_shards(3, [[(0, "a"), (1, "b")]])  # problem 2 missing
    with pytest.raises(ValueError):
        sweep.merge_shards(2, [[(0, "a"), (1, "b")], [(1, "c")]])  # reported twice
    with pytest.raises(ValueError):
        sweep.shard(4, 2, 2)


def test_reference_arm_other_ranks_exit_quietly(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        warmup, steps, gpus, ref_iters = 3, 2, 2, 80

    assert bench.run_reference(Args(), bench.problem_config(32)) == 0
    assert capsys.readouterr().out == ""
