"""bench.py's multi-process plumbing on the host (gloo, world size 2): rank setup from
torchrun's environment, the max-over-ranks timing reduction, the largest-first sharding
of the batched sweep, and the reference arm running on rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    try:
        got_ws, got_rank, local = bench.dist_setup("gloo")
        m = bench.allreduce_max(1.5 + rank, got_ws)
        bench.barrier(got_ws)
        from retainwall_code_b200 import cases as C

        specs = C.batch_sweep(n_cases=64, seed=5)
        owner, loads = bench.shard_cases(specs, got_ws)
        q.put((got_rank, got_ws, m, owner, loads))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert all(r[2] == 2.5 for r in res)  # max over ranks
    owner0, loads0 = res[0][3], res[0][4]
    assert owner0 == res[1][3]  # every rank derives the same partition
    assert set(owner0) == {0, 1} and len(owner0) == 64
    assert max(loads0) / min(loads0) < 1.05  # largest-first packing balances the soil


def test_shard_cases_is_a_partition():
    sys.path.insert(0, ROOT)
    import bench
    from retainwall_code_b200 import cases as C

    specs = C.batch_sweep(n_cases=64, seed=5)
    for ws in (1, 2, 4, 8):
        owner, loads = bench.shard_cases(specs, ws)
        sizes = [s["nx"] * s["ny"] * s["nz"] for s in specs]
        assert sum(loads) == sum(sizes)
        for r in range(ws):
            assert loads[r] == sum(n for n, o in zip(sizes, owner) if o == r)
        assert max(loads) - min(loads) <= max(sizes)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        workload, steps, warmup = "wall2", 1, 3

    bench.run_reference(Args(), 2, 1)  # rank 1 of 2: no work, no output
    assert capsys.readouterr().out == ""
