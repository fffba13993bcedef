"""The multi-GPU benchmark path runs independent replicas (the step does not
shard) and reports the whole-job rate over the slowest rank's time.  Its
host-side reduction is exercised here with two gloo ranks on the CPU, and so
is failure detection: a rank whose step fails leaves, and the other learns of
it from the collective's error within the process-group time-out."""
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
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    rate = bench.whole_job_rate(1000, 20, world, ms)
    q.put((rank, ms, rate))
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[0][2] == pytest.approx(1000 * 20 * 2 / 0.015)


def _failing_worker(rank, world, port, q):
    """rank 1 fails its step on the host (an exception before the timing
    collective) and leaves; rank 0 must learn of it from the collective with
    an error, not wait for ever"""
    import datetime
    import time
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        q.put((1, "failed step", 0.0))
        return  # leaves without taking part in the collective
    t0 = time.time()
    try:
        bench.max_over_ranks(10.0, dist, "cpu")
        q.put((0, "no error", time.time() - t0))
    except Exception as ex:  # noqa: BLE001 - any error is the expected outcome
        q.put((0, type(ex).__name__, time.time() - t0))


def test_a_failed_replica_is_reported_not_waited_for():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r[0], r[1:]) for r in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
    assert res[1][0] == "failed step"
    assert res[0][0] != "no error"
    assert res[0][1] < 60.0
