"""Multi-process plumbing of bench.py on the CPU (gloo, world_size 2).

The solver shards as independent replicas: each rank solves its own batch and the
only collectives are the timing barrier and the max-over-ranks reduction of the
timed region.  These run here as two gloo ranks.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, lr = bench.dist_env()
        assert (r, w, lr) == (rank, world, rank)
        bench.barrier(None)
        # each rank reports a different timed-region length; every rank must see the max
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank)
        bench.barrier(None)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_single_process_is_identity():
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.dist_env()[1] >= 1


def test_reference_arm_runs_on_rank0_only(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr("sys.argv", ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"])
    bench.main()  # rank 1 exits without work and prints nothing
    assert capsys.readouterr().out == ""


@pytest.mark.parametrize("n", [1, 2])
def test_value_is_whole_job_throughput(n):
    # value = all ranks' instances / max time: n replicas of B instances in T seconds
    B, steps, total_ms = 4096, 5, 1000.0
    assert n * B * steps / (total_ms * 1e-3) == pytest.approx(n * 20480.0)
