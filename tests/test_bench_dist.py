"""The multi-GPU path of bench.py on CPU: two gloo ranks (127.0.0.1), each a replica with
its own seeds; the timed value is the max over ranks; the reference leg runs on rank 0
only.  No GPU is touched."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    import bench
    w, r, local = bench.dist_setup()
    vmax = bench.reduce_max(1.5 + r, w, "cpu")
    seeds = bench.replica_seeds(r)
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, w, local, vmax, seeds))


def test_two_gloo_ranks_reduce_max_and_distinct_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 for x in res)
    assert all(x[3] == pytest.approx(2.5) for x in res)          # max over ranks on every rank
    assert res[0][4] != res[1][4]                                  # replicas solve different systems


def test_reference_leg_runs_on_rank_zero_only(capsys, monkeypatch):
    import sys
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        gpus, steps, warmup = 2, 1, 0
    bench.run_reference(Args, 2, 1)      # rank 1: returns at once, prints nothing
    assert capsys.readouterr().out == ""
