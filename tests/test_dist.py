"""N>1 host logic of the replica runs, with gloo ranks on the CPU (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    from edrixs_b200 import dist
    ws, r = dist.init_from_env(backend="gloo", timeout_s=60)
    dist.barrier()
    # each rank "measured" a different elapsed time; the job time is the slowest rank's
    m = dist.reduce_max(1.5 + r)
    q.put((r, ws, m))
    dist.finalize()


def test_replica_timing_reduction_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    out = sorted(q.get(timeout=5) for _ in range(2))
    assert out == [(0, 2, 2.5), (1, 2, 2.5)]
    assert all(p.exitcode == 0 for p in procs)


def test_single_rank_is_plain():
    from edrixs_b200 import dist
    assert dist.reduce_max(3.25) == 3.25
    dist.barrier()


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_nonzero_ranks_exit_quietly(rank, monkeypatch, capsys):
    """bench.py --impl reference: only rank 0 runs and prints; other ranks exit 0."""
    import bench
    monkeypatch.setenv("RANK", str(rank))
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        nbath, nelec, steps, warmup, nkryl = 10, 10, 1, 0, 150
    bench.run_reference(A())
    assert capsys.readouterr().out == ""
