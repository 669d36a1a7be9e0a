"""Host-side logic of the server and the autotuner (no GPU)."""
import pytest

from tomogpi_b200.autotune import extrapolate, first_views, pick
from tomogpi_b200.config import ConfigCT
from tomogpi_b200.serve import DEFAULT_LANES, HBMPool, lane_index, lane_shares, poisson_stream


def test_pool_accounting():
    p = HBMPool(100)
    assert p.fits(60)
    p.take(60)
    assert not p.fits(50) and p.fits(40)
    with pytest.raises(MemoryError):
        p.take(50)
    p.give(60)
    assert p.used == 0


def test_poisson_stream_is_seeded_and_weighted():
    mk = lambda rid, n, t: (rid, n, t)  # noqa: E731
    a = poisson_stream(7, 400, 10.0, [128, 256, 512, 768, 1024], [0.3, 0.3, 0.2, 0.15, 0.05], mk)
    b = poisson_stream(7, 400, 10.0, [128, 256, 512, 768, 1024], [0.3, 0.3, 0.2, 0.15, 0.05], mk)
    assert a == b
    times = [x[2] for x in a]
    assert all(t2 > t1 for t1, t2 in zip(times, times[1:]))
    assert 30 < times[-1] < 50  # 400 arrivals at 10 Hz
    frac_small = sum(1 for x in a if x[1] in (128, 256)) / len(a)
    assert 0.5 < frac_small < 0.7


def test_tuner_helpers():
    c = ConfigCT.cone_beam(32, 360)
    sub = first_views(c, 12)
    assert sub.projection_nb == 12
    assert abs(sub.phi()[5] - c.phi()[5]) < 1e-12
    assert pick({"rs_tex": 3.0, "rs_cell8": 2.0, "vi_zc1": 5.0, "vi_zc2": 4.0}) == \
        {"rs_layout": "cell8", "vi_zc": 2, "vi_layout": "padded"}
    assert pick({"rs_tex": 3.0, "vi_zc1": 5.0, "vi_zc2": 4.0, "vi_tma": 3.5})["vi_layout"] == "tma"


def test_lane_classes_and_shares():
    assert [lane_index(DEFAULT_LANES, ConfigCT.cone_beam(n, n)) for n in (64, 128, 256, 384, 512, 768, 1024)] == \
        [0, 0, 0, 1, 1, 2, 2]
    assert lane_shares([False, False, False]) == [1.0, 1.0, 1.0]
    assert lane_shares([False, True, False]) == [1.0, 1.0, 1.0]   # alone: the whole GPU
    assert lane_shares([True, False, True]) == [1.0, 1.0, 0.5]    # smallest busy lane takes free slots
    assert lane_shares([True, True, True]) == [1.0, 1 / 3, 1 / 3]
    assert lane_shares([False, True, True]) == [1.0, 1.0, 0.5]


def test_tuner_extrapolation():
    # fixed cost 4 ms + 0.5 ms per view: trials over 16 and 32 views predict 512 views
    assert abs(extrapolate(4 + 0.5 * 16, 4 + 0.5 * 32, 16, 512) - (4 + 0.5 * 512)) < 1e-9


def test_latency_percentiles_need_enough_results():
    from tomogpi_b200.serve import Result, latency_percentiles

    res = [Result(i, None, arrival=float(i), admitted=float(i) + 0.5, finished=float(i) + 1.0 + (i == 7) * 9.0,
                  footprint=1) for i in range(20)]
    small = latency_percentiles(res)
    assert small["n"] == 20 and small["p99_ms"] is None and small["max_ms"] == 10000.0
    assert small["p50_ms"] == 1000.0 and small["queue_p50_ms"] == 500.0 and small["service_p50_ms"] == 500.0
    many = latency_percentiles(res * 5)
    assert many["n"] == 100 and many["p99_ms"] is not None and many["p99_ms"] <= many["max_ms"]
