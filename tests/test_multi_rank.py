"""Multi-rank host logic of the replica form over gloo on CPU (world size 2): the job
assignment every rank computes alone, the max-over-ranks device time, and rank 0 gathering
the served results of both ranks."""
import multiprocessing as mp
import os
import socket

import pytest

from tomogpi_b200.replicas import assign_jobs, dist_env


def test_assignment_is_deterministic_and_balanced():
    works = [5, 1, 9, 3, 3, 8, 2, 7]
    a = assign_jobs(works, 3)
    assert a == assign_jobs(works, 3)
    assert sorted(j for part in a for j in part) == list(range(len(works)))
    loads = [sum(works[j] for j in part) for part in a]
    assert max(loads) - min(loads) <= max(works)
    assert assign_jobs(works, 1) == [list(range(len(works)))]
    assert assign_jobs([], 2) == [[], []]
    with pytest.raises(ValueError):
        assign_jobs(works, 0)


def test_dist_env_defaults(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert dist_env() == (1, 0, 0)
    monkeypatch.setenv("WORLD_SIZE", "4")
    monkeypatch.setenv("RANK", "2")
    monkeypatch.setenv("LOCAL_RANK", "2")
    assert dist_env() == (4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    try:
        from tomogpi_b200.replicas import max_over_ranks, serve_replicated

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        t = max_over_ranks(10.0 + rank)
        reqs = [{"rid": i, "work": w} for i, w in enumerate([4, 1, 3, 2, 6, 5])]
        served = []

        def serve(mine):
            served.extend(r["rid"] for r in mine)
            return [(r["rid"], rank) for r in mine]

        res = serve_replicated(reqs, lambda r: r["work"], serve)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, t, served, res))
    except Exception as e:  # reported to the parent, never swallowed
        q.put((rank, "error", repr(e), None))


def test_two_gloo_ranks_time_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, t, served, res = q.get(timeout=120)
        out[rank] = (t, served, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        assert out[rank][0] == 11.0, out[rank]          # max over ranks of 10 + rank
    assert out[1][2] is None                            # only rank 0 holds the results
    got = sorted(out[0][2])
    assert [rid for rid, _ in got] == list(range(6))    # every request served exactly once
    assert set(out[0][1]).isdisjoint(out[1][1])
    assert {rid for rid, rk in got if rk == 0} == set(out[0][1])
    assert sorted(out[0][1] + out[1][1]) == list(range(6))
