"""bench.py's multi-GPU form runs independent replicas, one per rank, and
reports all ranks' work over the slowest rank's time. The reduction is
exercised here with two gloo ranks on CPU (no GPU)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as tdist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [120.0, 180.0][rank]  # rank 1 is the slow replica
    worst = bench.max_over_ranks(ms)
    q.put((rank, worst, bench.replica_rate(20, worst, world)))
    tdist.barrier()
    tdist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, worst, rate in got:
        assert worst == 180.0
        assert rate == pytest.approx(2 * 20 / 0.180)


def test_single_process_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(42.0) == 42.0
    assert bench.replica_rate(20, 500.0, 1) == pytest.approx(40.0)


def test_per_pass_rates_against_the_peaks():
    sys.path.insert(0, ROOT)
    import bench
    alg = 2 * 16 * 2 ** 30
    d = bench.per_pass_gbs(alg, [10.0, 20.0, 0.0, 5.0], 6548.8)
    assert d["passes"] == 3  # a zero duration is dropped
    assert d["median"] == pytest.approx(alg / 0.010 / 1e9)
    assert d["min"] < d["median"] < d["max"]
    assert d["median_frac"] == pytest.approx(d["median"] / 6548.8)
    assert d["median_frac_of_nominal"] == pytest.approx(d["median"] / 8000.0)
    assert bench.per_pass_gbs(alg, [], 1.0) is None
