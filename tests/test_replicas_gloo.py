"""The N > 1 path of bench.py on the CPU: independent replicas whose only
communication is the aggregation after the timed region (slowest rank's
time, summed iterations), run as two gloo ranks over 127.0.0.1.

* Both ranks get the same job figures.
* A rank that leaves before the collective makes the other fail within the
  process-group timeout instead of waiting for ever.
"""
import datetime
import socket

import pytest
import torch.multiprocessing as mp

from tealeaf_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _init(rank, world, port, timeout_s):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _aggregate_worker(rank, world, port, q):
    dist = _init(rank, world, port, 30)
    ms, its = 100.0 + 50.0 * rank, 1000 + rank
    mx, sm = replicas.aggregate(ms, its, world, device="cpu")
    thr = replicas.throughput(ms, its, world, device="cpu")
    q.put((rank, mx, sm, thr))
    dist.barrier()
    dist.destroy_process_group()


def _leaver_worker(rank, world, port, q):
    dist = _init(rank, world, port, 5)
    if rank == 1:
        q.put((rank, "left"))
        return   # never reaches the collective
    try:
        replicas.aggregate(100.0, 1000, world, device="cpu")
        q.put((rank, "completed"))
    except Exception as exc:   # the peer is gone: an error, not a hang
        q.put((rank, "error: " + type(exc).__name__))


def _run(target, world=2, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0])


def test_single_rank_is_identity():
    assert replicas.aggregate(12.5, 40, 1) == (12.5, 40.0)
    assert replicas.throughput(500.0, 100, 1) == pytest.approx(200.0)


def test_two_gloo_ranks_aggregate_slowest_time_and_summed_work():
    out = _run(_aggregate_worker)
    for rank, mx, sm, thr in out:
        assert mx == 150.0 and sm == 2001.0
        assert thr == pytest.approx(2001.0 / 0.150)


def test_rank_that_leaves_fails_the_other_within_the_timeout():
    out = _run(_leaver_worker, timeout=90)
    assert out[1] == (1, "left")
    assert out[0][1].startswith("error"), out[0]
