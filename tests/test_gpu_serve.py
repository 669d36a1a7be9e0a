"""Continuous-batching server: requests arriving over time are admitted by HBM footprint,
overlap on the device, and each result is the same as running the job alone."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _request(rid, n, arrival, views=None):
    import oracle
    from tomogpi_b200 import ConfigCT, phantoms
    from tomogpi_b200.serve import Request

    cfg = ConfigCT.cone_beam(n, views or n, magnification=1.5 + (rid % 5) * 0.25)
    truth = oracle.phantom(phantoms.random_ellipsoids(100 + rid, 6, n), n, n, n)
    g = oracle.project(cfg, oracle.SIDDON, truth)
    g = g + np.random.default_rng(rid).normal(0, 0.01 * g.max(), g.shape).astype(np.float32)
    return Request(rid, cfg, g.astype(np.float32), arrival)


def _alone(req, params):
    import tomogpi_b200 as t

    b = t.Batch(params)
    vol = torch.zeros(req.cfg.volume_shape, device="cuda:0")
    g = torch.from_numpy(req.sinogram).cuda()
    b.add(req.cfg, vol, g, rs_layout="tex")
    b.iterate(params.gradient_iteration_nb)
    out = vol.cpu().numpy()
    b.close()
    return out


def test_served_results_equal_alone_and_overlap():
    import tomogpi_b200 as t
    from tomogpi_b200.serve import Server, latency_percentiles

    params = t.GradientParams(gradient_iteration_nb=4, optimal_step_iteration_nb=5)
    reqs = [_request(i, n, 0.002 * i) for i, n in enumerate([24, 16, 32, 24, 16, 40])]
    srv = Server(params)
    res = srv.run(reqs)
    srv.close()
    assert sorted(r.rid for r in res) == list(range(len(reqs)))
    for r in res:
        assert np.array_equal(r.volume.numpy(), _alone(reqs[r.rid], params)), r.rid
    spans = sorted((r.admitted, r.finished) for r in res)  # several jobs were live at once
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    pct = latency_percentiles(res)
    assert pct["n"] == len(reqs) and pct["p99_ms"] is None  # too few results for a 99th percentile
    assert 0 < pct["p50_ms"] <= pct["max_ms"]
    assert pct["queue_p50_ms"] >= 0 and pct["service_p50_ms"] > 0


def test_admission_respects_the_hbm_budget():
    import tomogpi_b200 as t
    from tomogpi_b200.serve import Server, job_footprint

    params = t.GradientParams(gradient_iteration_nb=3, optimal_step_iteration_nb=4, storage="bf16")
    reqs = [_request(i, 32, 0.0) for i in range(5)]
    for r in reqs:
        r.tuning = {"rs_layout": "cell8", "vi_zc": 2}
    one = job_footprint(reqs[0].cfg, params, reqs[0].tuning)
    srv = Server(params, hbm_budget=int(2.5 * one))  # at most two jobs at a time
    res = srv.run(reqs)                                 # HBMPool.take raises beyond the budget
    srv.close()
    assert srv.peak_live == 2 and len(res) == 5 and srv.pool.used == 0


def test_lanes_overlap_and_results_equal_alone():
    """Jobs of two size classes in two lanes (two batches on two streams, SMs split by the
    CTA shares) run at the same time, and each result is bit-identical to the job alone."""
    import tomogpi_b200 as t
    from tomogpi_b200.serve import LaneSpec, Server

    params = t.GradientParams(gradient_iteration_nb=4, optimal_step_iteration_nb=5)
    reqs = [_request(i, n, 0.001 * i, views=v) for i, (n, v) in
            enumerate([(48, 96), (16, 24), (24, 24), (16, 32), (40, 64), (24, 16)])]
    lanes = (LaneSpec("small", 24.0 ** 4), LaneSpec("large", float("inf")))
    srv = Server(params, lanes=lanes)
    res = srv.run(reqs)
    srv.close()
    assert sorted(r.rid for r in res) == list(range(len(reqs)))
    by_lane = {}
    for r in res:
        assert np.array_equal(r.volume.numpy(), _alone(reqs[r.rid], params)), r.rid
        by_lane.setdefault(r.lane, []).append(r)
    assert set(by_lane) == {"small", "large"}
    big = by_lane["large"][0]
    assert any(s.admitted < big.finished and s.finished > big.admitted for s in by_lane["small"])


@pytest.mark.parametrize("share", [0.001, 0.3])
def test_reduced_cta_share_same_result(share):
    """A batch whose persistent launches may use only a few CTAs (down to one) computes the
    same iterates."""
    import tomogpi_b200 as t

    params = t.GradientParams(gradient_iteration_nb=3, optimal_step_iteration_nb=4, storage="bf16")
    req = _request(7, 32, 0.0)
    ref = None
    for sh in (1.0, share):
        b = t.Batch(params)
        b.set_share(sh)
        vol = torch.zeros(req.cfg.volume_shape, device="cuda:0")
        g = torch.from_numpy(req.sinogram).cuda().to(torch.bfloat16)
        b.add(req.cfg, vol, g, rs_layout="cell8")
        b.iterate(3)
        out = vol.cpu().numpy()
        b.close()
        if ref is None:
            ref = out
    assert np.array_equal(out, ref)


def test_autotuner_picks_and_caches(tmp_path, monkeypatch):
    import tomogpi_b200.autotune as at
    from tomogpi_b200 import ConfigCT

    monkeypatch.setattr(at, "_CACHE", tmp_path / "tune.json")
    monkeypatch.setattr(at, "_mem", None)
    cfg = ConfigCT.cone_beam(48, 64)
    r = at.tune(cfg, "f32", trial_views=4)
    assert r["rs_layout"] in ("tex", "hybrid", "march", "cell8", "plain") and r["vi_zc"] in (1, 2, 4)
    assert set(r["trials"]) == {"rs_tex", "rs_hybrid", "rs_march", "rs_cell8", "rs_plain", "vi_zc1", "vi_zc2",
                                "vi_zc4", "vi_tma"}
    assert (tmp_path / "tune.json").exists() and at.tune(cfg, "f32") == r
