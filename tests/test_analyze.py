"""CPU checks of the TTS99 estimators (reference gpu/onsager_v2_20261007/src/analyze.py:15-88) on synthetic run files."""
import json
import math

import pytest

from anechoic_b200 import analyze as Z


def test_wilson_interval_properties():
    for n in (1, 7, 100, 4096):
        for k in sorted({0, 1, n // 3, n - 1, n}):
            lo, hi = Z.wilson(k, n)
            assert 0.0 <= lo <= k / n + 1e-12 and k / n - 1e-12 <= hi <= 1.0
            lo2, hi2 = Z.wilson(n - k, n)
            assert math.isclose(lo, 1.0 - hi2, abs_tol=1e-12) and math.isclose(hi, 1.0 - lo2, abs_tol=1e-12)
    assert Z.wilson(0, 0) == (0.0, 1.0)
    # closed form at k = 0: upper bound z^2 / (n + z^2)
    n = 50
    assert math.isclose(Z.wilson(0, n)[1], Z.Z95 ** 2 / (n + Z.Z95 ** 2), rel_tol=1e-12)


def test_tts_formulas():
    assert Z.tts99(1.0, 3.0) == 3.0 and Z.tts99(0.0, 3.0) == math.inf
    assert math.isclose(Z.tts99(0.5, 2.0), 2.0 * math.log(0.01) / math.log(0.5))
    assert Z.tts99_secondary(0.0, 8, 1.0) == math.inf and Z.tts99_secondary(1.0, 8, 1.0) == 0.0
    # secondary with B anneals per batch equals primary with P = 1 - (1 - p)^B
    p, B, t = 0.01, 64, 5.0
    assert math.isclose(Z.tts99_secondary(p, B, t), Z.tts99(1 - (1 - p) ** B, t), rel_tol=1e-9)
    assert Z.tts99_whole(0.5, 2.0) == 2.0 * math.ceil(math.log(0.01) / math.log(0.5))


def test_estimate_from_run_files(tmp_path):
    prefix = str(tmp_path / "run")
    bat = [dict(batch=b, chains=16, trial_offset=16 * b, device_ms=2.0 + 0.5 * b, host_ms=3.0, successes=s)
           for b, s in enumerate([0, 2, 1, 0])]
    with open(prefix + ".batches.jsonl", "w") as f:
        for b in bat:
            f.write(json.dumps(b) + "\n")
    with open(prefix + ".summary.json", "w") as f:
        json.dump(dict(chains=16, batches=4, steps=100, t0=30.0, t1=5.0, q=4.0, ramp=True, cut_mismatches=0), f)
        f.write("\n")
    e = Z.estimate(prefix)
    assert e["B"] == 16 and e["batches"] == 4 and e["successes"] == 3 and e["trials"] == 64
    assert e["P_batch"] == 0.5 and math.isclose(e["p"], 3 / 64)
    assert math.isclose(e["t_batch_ms"], 2.75)
    assert math.isclose(e["tts_primary_ms"], Z.tts99(0.5, 2.75))
    lo, hi = e["tts_primary_ci_ms"]
    assert lo <= e["tts_primary_ms"] <= hi
    assert Z.selection_score(e, "primary") >= e["tts_primary_ms"]


def _dec(v):
    if v == "inf":
        return math.inf
    if isinstance(v, list):
        return [_dec(x) for x in v]
    return v


def _same(a, b):
    if isinstance(a, list):
        return len(a) == len(b) and all(_same(x, y) for x, y in zip(a, b))
    if isinstance(a, float) or isinstance(b, float):
        if math.isinf(a) or math.isinf(b):
            return a == b
        return math.isclose(a, b, rel_tol=1e-12, abs_tol=1e-15)
    return a == b


def test_estimates_match_reference_fixture(tmp_path):
    """The reference's estimate() / selection_score() (gpu/onsager_v2_20261007/src/analyze.py:56-88) ran on run files
    in this CLI's format (tests/golden/make_analyze_golden.py); the same files give the same value for every field
    here. Where the reference raises (a cohort without successes: its Wilson bound reaches log(1 - P) = 0), this
    estimator returns an unbounded time to solution instead."""
    import os
    from tests.conftest import GOLDEN
    with open(os.path.join(GOLDEN, "analyze_estimates.json")) as f:
        cases = json.load(f)["cases"]
    assert len(cases) >= 6
    for c in cases:
        prefix = str(tmp_path / c["name"])
        with open(prefix + ".summary.json", "w") as f:
            f.write(c["summary"])
        with open(prefix + ".batches.jsonl", "w") as f:
            f.write(c["batches"])
        e = Z.estimate(prefix)
        e["selection_primary"] = Z.selection_score(e, "primary")
        e["selection_secondary"] = Z.selection_score(e, "secondary")
        if "raises" in c:
            assert e["successes"] == 0 and e["tts_primary_ms"] == math.inf and e["tts_secondary_ms"] == math.inf
            assert e["tts_primary_ci_ms"][1] == math.inf and e["selection_primary"] == math.inf
            continue
        for k, v in c["expected"].items():
            assert k in e, (c["name"], k)
            assert _same(_dec(v), e[k]), (c["name"], k, v, e[k])
