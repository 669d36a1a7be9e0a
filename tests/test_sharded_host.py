"""Host logic of the view-split reconstruction (tomogpi_b200/sharded.py) over gloo on CPU:
the view partition, and the exchange protocol of iterate_exchange on a small dense
least-squares problem whose rows (views) are split over two ranks, against one rank."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from tomogpi_b200.sharded import PHASE_GRADIENT, PHASE_NORMS, PHASE_UPDATE, iterate_exchange, view_ranges


def test_view_ranges():
    assert view_ranges(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert view_ranges(8, 1) == [(0, 8)]
    assert sum(c for _, c in view_ranges(513, 8)) == 513
    with pytest.raises(ValueError):
        view_ranges(3, 4)
    with pytest.raises(ValueError):
        view_ranges(3, 0)


def _toy(rows, torch):
    """A toy 'solver' with the phase semantics of tomo_solver_phase for f <- f + alpha dJ,
    dJ = -2 H^T (g - H f), alpha = -||dJ||^2 / (2 ||H dJ||^2) while it < opt, else alpha_min."""
    rng = np.random.default_rng(1)
    H = torch.tensor(rng.normal(size=(12, 5)), dtype=torch.float64)
    g = torch.tensor(rng.normal(size=12), dtype=torch.float64)
    Hk, gk = H[rows], g[rows]
    state = {"f": torch.zeros(5, dtype=torch.float64), "amin": -1e30, "alphas": []}
    dJ = torch.zeros(5, dtype=torch.float64)
    norms = torch.zeros(8, dtype=torch.float64)

    def phase(it, bits, opt_nb=4):
        f = state["f"]
        if bits & PHASE_GRADIENT:
            dJ.copy_(-2.0 * Hk.T @ (gk - Hk @ f))
        if bits & PHASE_NORMS and it < opt_nb:
            norms[0] = float(dJ @ dJ)
            norms[1] = float((Hk @ dJ) @ (Hk @ dJ))
            norms[2] = 7.0          # a norm of the summed dJ: must count once, not once per rank
        if bits & PHASE_UPDATE:
            if it < opt_nb:
                a = -norms[0].item() / (2.0 * norms[1].item())
                state["amin"] = max(a, state["amin"])
            else:
                a = state["amin"]
            state["alphas"].append(a)
            f += a * dJ

    return phase, dJ, norms, state


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        rows = list(range(12))[rank * 6:(rank + 1) * 6]
        phase, dJ, norms, state = _toy(rows, torch)
        iterate_exchange(phase, dJ, norms, 1, 7, 4, lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM), rank)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, state["f"].numpy().tolist(), state["alphas"], float(norms[2])))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), None))


def test_two_gloo_ranks_match_one_rank():
    import torch

    phase, dJ, norms, state = _toy(list(range(12)), torch)
    iterate_exchange(phase, dJ, norms, 1, 7, 4, None)
    ref_f, ref_a = state["f"].numpy(), state["alphas"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, f, a, n2 = q.get(timeout=120)
        assert f != "error", a
        out[rank] = (np.array(f), a, n2)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(out[0][0], out[1][0])
    assert np.allclose(out[0][0], ref_f, rtol=1e-12, atol=1e-12)
    assert np.allclose(out[0][1], ref_a, rtol=1e-12)
    assert out[0][2] == 7.0 and out[1][2] == 7.0


def test_default_device_from_local_rank(monkeypatch):
    from tomogpi_b200.sharded import default_device

    monkeypatch.setenv("LOCAL_RANK", "3")
    assert default_device(rank=11, device_count=8) == 3
    monkeypatch.delenv("LOCAL_RANK")
    assert default_device(rank=2, device_count=4) == 2
    with pytest.raises(ValueError, match="no GPU on this node"):
        default_device(rank=9, device_count=8)  # a global rank of a multi-node run
    monkeypatch.setenv("LOCAL_RANK", "8")
    with pytest.raises(ValueError):
        default_device(rank=0, device_count=8)
