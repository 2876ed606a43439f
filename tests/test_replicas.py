"""Replica placement of jobs over GPUs (one process per GPU): partition and the end-of-run merge, run as two
gloo ranks on CPU (the data path has no collective; only this merge exchanges anything)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mycel_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, jobs, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = replicas.partition(jobs, rank, world)
    # a stand-in for the rank's server: latency = job size / 100, one SIMP iteration per job
    local = {"latencies": [j / 100.0 for j in mine], "simp_iterations": len(mine),
             "first_submit_s": 0.0 + rank, "last_finish_s": 10.0 + rank}
    merged = replicas.merge(local)
    q.put((rank, mine, merged))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_covers_each_job_once():
    jobs = list(range(11))
    shares = [replicas.partition(jobs, r, 3) for r in range(3)]
    assert sorted(x for s in shares for x in s) == jobs
    assert shares[0] == [0, 3, 6, 9] and shares[2] == [2, 5, 8]
    with pytest.raises(ValueError):
        replicas.partition(jobs, 3, 3)


def test_merge_single_process_matches_percentiles():
    out = replicas.merge({"latencies": [1.0, 2.0, 3.0, 4.0], "simp_iterations": 8, "first_submit_s": 0.0,
                          "last_finish_s": 4.0})
    assert out["p50_latency_s"] == 2.0 and out["p99_latency_s"] == 4.0 and out["simp_iter_s"] == 2.0


def test_two_gloo_ranks_merge_to_the_whole_stream():
    world, jobs = 2, list(range(1, 21))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, jobs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shares = [r[1] for r in res]
    assert sorted(shares[0] + shares[1]) == jobs and not set(shares[0]) & set(shares[1])
    whole = [j / 100.0 for j in jobs]
    for _rank, _mine, merged in res:
        assert merged["ranks"] == 2 and merged["completed"] == len(jobs)
        assert merged["p50_latency_s"] == replicas.percentile(whole, 0.5)
        assert merged["p99_latency_s"] == replicas.percentile(whole, 0.99)
        assert merged["simp_iterations"] == len(jobs)
        assert merged["simp_iter_s"] == len(jobs) / (11.0 - 0.0)
