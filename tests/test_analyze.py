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
