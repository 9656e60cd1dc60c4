"""The learned warm start's judgement, on the host: given the sweeps each start needed on the same twin steps, the
network is kept only in a mode that needs fewer sweeps than the carried impulses, in the better of its two modes,
with the gains and the ceiling reported as measured. The twin steps themselves run on a GPU
(tests/test_gpu_learned.py); here their result is given."""
import numpy as np
import pytest

from vxr import learned as Lm


def measured(carried, zero, network_all, network_new, ceiling=None):
    mean = {"carried": carried, "zero": zero, "network_all": network_all, "network_new": network_new}
    if ceiling:
        mean.update(ceiling)
    return {"samples": 3, "lead_steps": 2, "tolerance_m": 1e-4, "cap": 64, "mean_sweeps": mean,
            "reached": {k: 0.5 for k in mean}, "by_substep": {k: [v] * 4 for k, v in mean.items()},
            "pairs_alone_by_substep": {k: [v] * 4 for k, v in mean.items()},
            "walls_alone_by_substep": {k: [v / 2] * 4 for k, v in mean.items()},
            "gain_vs_carried": {k: carried / v for k, v in mean.items()},
            "answers": {"tolerance_m": 1e-6, "cap": 256}, "twins_aligned": True}


@pytest.fixture
def given(monkeypatch):
    def use(result):
        monkeypatch.setattr(Lm, "compare_starts", lambda *a, **k: result)
    return use


def test_the_network_is_dropped_when_no_mode_needs_fewer_sweeps(given):
    given(measured(50.0, 54.0, 54.0, 50.0))
    v = Lm.judge({}, [], net=object())
    assert v["kept"] is False and v["mode"] == 0
    assert v["fallback"].startswith("plain warm start")
    assert v["gain_vs_warm_start"] == pytest.approx(1.0)


@pytest.mark.parametrize("network_all, network_new, mode", [(40.0, 45.0, 2), (45.0, 40.0, 3), (44.0, 44.0, 2)])
def test_the_network_is_kept_in_its_better_mode(given, network_all, network_new, mode):
    given(measured(50.0, 60.0, network_all, network_new))
    v = Lm.judge({}, [], net=object())
    assert v["kept"] is True and v["mode"] == mode and v["fallback"] is None
    best = min(network_all, network_new)
    assert v["gain_vs_warm_start"] == pytest.approx(50.0 / best)
    assert v["gain_vs_cold_start"] == pytest.approx(60.0 / best)
    assert v["plain_warm_start"] == 50.0 and v["plain_cold_start"] == 60.0


def test_the_ceiling_is_reported_as_measured(given):
    ceiling = {k: 40.0 for k in Lm.CEILING_STARTS}
    given(measured(50.0, 52.0, 51.0, 50.5, ceiling))
    v = Lm.judge({}, [], net=object(), ceiling=True)
    assert set(v["ceiling"]["mean_sweeps"]) == set(Lm.CEILING_STARTS)
    assert v["ceiling"]["gain_vs_carried"]["first_whole_all"] == pytest.approx(1.25)
    assert v["ceiling"]["twins_aligned"] is True
    assert set(v["same_steps"]["by_substep"]) >= set(Lm.NETWORK_STARTS)


def test_rows_in_order_ignores_the_order_within_a_round():
    rng = np.random.default_rng(3)
    f = rng.standard_normal((40, 16)).astype(np.float32)
    g = f[rng.permutation(40)]
    assert np.array_equal(Lm.rows_in_order(f), Lm.rows_in_order(g))
    h = g.copy()
    h[5, 3] = np.nextafter(h[5, 3], np.float32(np.inf))
    assert not np.array_equal(Lm.rows_in_order(f), Lm.rows_in_order(h))
