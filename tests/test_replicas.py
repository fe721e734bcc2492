"""The N > 1 path of bench.py on CPU: two ranks over gloo.

The workload does not shard (replicas only): each rank runs its own copy and
the ranks meet only to synchronise the timed region and take the maximum of
their times.  These tests run that plumbing with world size 2 on CPU, and the
reference arm's rank handling (rank 0 works and prints, the others exit 0)."""

import multiprocessing as mp
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    try:
        import bench
        d = bench._Dist(ws, rank, rank, "gloo")
        d.barrier()
        m = d.max(10.0 * (rank + 1))
        d.barrier()
        d.close()
        q.put((rank, m))
    except Exception as e:  # pragma: no cover - reported through the queue
        q.put((rank, repr(e)))


def test_two_rank_barrier_and_max():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the maximum over ranks
    assert out == {0: 20.0, 1: 20.0}


def _ref_rank(rank, ws, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    q.put((rank, bench.main(["--impl", "reference", "--steps", "1", "--warmup", "1"])))


def test_reference_arm_other_ranks_exit_without_work():
    """Only rank 0 of the reference arm runs the CPU port; rank 1 returns 0
    at once (checked without running rank 0's workload)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_rank, args=(1, 2, q))
    p.start()
    rank, rc = q.get(timeout=120)
    p.join(timeout=60)
    assert (rank, rc, p.exitcode) == (1, 0, 0)


@pytest.mark.parametrize("ws", [1, 2])
def test_workload_config_is_rank_independent(ws):
    sys.path.insert(0, ROOT)
    import bench
    c = bench.workload_config(ws)
    assert c == bench.workload_config(ws)
    assert c["bytes_per_step"] == 565632064
    assert c["parallelism"] == ("replicas" if ws > 1 else "single")
