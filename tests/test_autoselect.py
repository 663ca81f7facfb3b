"""engine="auto": the cost model that picks an engine per launch, against device times measured on a B200
(tests/golden/engine_times_b200.json, written by tests/golden/make_engine_times.py), and on the GPU the flip fraction
it learns from each run. The engines' results are bit-identical, so the choice only moves the time."""
import json
import math
import os

import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "engine_times_b200.json")


def _cases():
    with open(FIX) as f:
        return json.load(f)["cases"]


def _estimate(c):
    return A.auto_estimate(c["n"], c["kbits"], c["chains"], c["S"], c["flip_fraction"], c["per_wave"], fp4=c["fp4"])


def test_picks_near_the_fastest_engine():
    """With the flip fraction a run saw, the model's pick is within 20% of the fastest measured engine in every
    case (6% measured), and within 3% over the geometric mean of all cases (0.2% measured)."""
    logs = []
    for c in _cases():
        est = _estimate(c)
        best = min(c["ms"].values())
        got = c["ms"][est["pick"]]
        assert got <= 1.2 * best, (c["case"], c["sched"], c["chains"], est, c["ms"])
        logs.append(math.log(got / best))
    assert math.exp(sum(logs) / len(logs)) < 1.03


def test_estimates_track_measured_times():
    """Each engine's estimate is within a factor 2 of its measured device time, and within 1.4 for 95% of the
    launches (the fit spans n = 500 ... 10000, 1- to 4-bit couplings, flip fractions 0.03 ... 0.47). The largest miss
    is the plain engine on 4-bit couplings with more than a hundred anneals under the counted-Onsager schedule, which
    slows with the number of anneals in flight (a 1000-spin instance: 13 ms for one anneal, 24 ms for 148)."""
    ratios = []
    for c in _cases():
        est = _estimate(c)
        for e, ms in c["ms"].items():
            r = est[e] / ms
            assert 1 / 2 < r < 2, (c["case"], c["sched"], c["chains"], e, est[e], ms)
            ratios.append(r)
    assert sum(1 / 1.4 < r < 1.4 for r in ratios) >= 0.95 * len(ratios)


def test_recorded_picks_match_the_model():
    """What the library picked on the GPU (after the measured runs) is what the host-only model computes."""
    for c in _cases():
        assert _estimate(c)["pick"] == c["auto_pick"], (c["case"], c["sched"], c["chains"])


def test_waves_and_availability():
    w = {"plain": 148, "tensor": 1152, "cluster": 15}
    one = A.auto_estimate(2000, 1, 15, 1000, 0.3, w, fp4=True)
    two = A.auto_estimate(2000, 1, 16, 1000, 0.3, w, fp4=True)
    assert two["cluster"] == pytest.approx(2 * one["cluster"]) and two["plain"] == one["plain"]
    # up to half an 8-CTA wave (7 anneals here) runs as one wave of 16-CTA clusters, at its own per-step cost
    small = [A.auto_estimate(2000, 1, c, 1000, 0.3, w, fp4=True)["cluster"] for c in (1, 7, 8)]
    assert small[0] == small[1] < small[2] == pytest.approx(one["cluster"])
    assert A.auto_estimate(2000, 1, 149, 1000, 0.3, w, fp4=True)["plain"] == pytest.approx(2 * one["plain"])
    sparse = A.auto_estimate(5000, 0, 64, 100, 0.1, {"plain": 148})
    assert sparse["pick"] == "plain" and set(sparse) == {"plain", "pick"}
    with pytest.raises(A.AncError):
        A.auto_estimate(2000, 1, 1, 100, 0.3, {})
    with pytest.raises(A.AncError):
        A.auto_estimate(2000, 3, 1, 100, 0.3, w)


@pytest.mark.gpu
def test_auto_learns_the_flip_fraction(cuda):
    """Before any run AUTO assumes a flip fraction of 0.25; after an AUTO run it uses the fraction that run saw on
    these tables and this instance (a few flips: the plain engine for 120 anneals); a caller's hint overrides; another
    instance starts from the prior again."""
    inst = I.complete_pm1(2000, 20261004)
    dev = A.DeviceInstance(inst)
    sc = dict(S=120, t0=15.0, q=8.0, kappa=2.0, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    ch = A.auto_choice(dev, tb, 120)
    assert ch["flip_fraction"] == pytest.approx(0.25)
    assert ch["per_wave"]["plain"] >= 148 and ch["per_wave"]["tensor"] >= 128 and ch["per_wave"]["cluster"] >= 1
    r = A.run(dev, tb, 7, 0, 120)
    phi = float(r.flips.sum()) / (120 * 2000 * sc["S"])
    ch = A.auto_choice(dev, tb, 120)
    assert ch["flip_fraction"] == pytest.approx(phi, abs=1e-6) and phi < 0.2
    assert ch["pick"] == "plain"
    assert A.run(dev, tb, 7, 120, 120).kernel == "plain"
    assert A.auto_choice(dev, tb, 120, flip_fraction=0.4)["pick"] == "tensor"
    assert A.run(dev, tb, 7, 240, 120, flip_fraction=0.4).kernel == "tensor-fp4"
    other = A.DeviceInstance(I.complete_pm1(1999, 5))
    assert A.auto_choice(other, tb, 120)["flip_fraction"] == pytest.approx(0.25)
