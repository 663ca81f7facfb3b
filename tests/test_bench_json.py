"""CPU: the bench line's helpers. TTS99 follows the reference's estimators (gpu/onsager_v2_20261007/src/analyze.py:
15-47). Non-finite values, such as TTS99 with no success at a short step budget, are written as null so the line
stays strict JSON."""
import json
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_tts99_estimators():
    t = 9.0
    assert bench.tts99(1.0, t) == t                                    # every batch succeeds: one batch
    assert bench.tts99(0.0, t) == math.inf
    assert math.isclose(bench.tts99(0.5, t), t * math.log(0.01) / math.log(0.5))
    B, p = 1024, 0.02
    assert math.isclose(bench.tts99_secondary(p, B, t), t * math.log(0.01) / (B * math.log(1 - p)))
    assert bench.tts99_secondary(0.0, B, t) == math.inf
    assert bench.tts99_secondary(1.0, B, t) == t / B                    # every anneal succeeds: one anneal's share


def test_line_is_strict_json():
    line = {"value": 1.5, "tts99_us": {"primary": math.inf, "secondary": float("nan")},
            "tts99_by_budget": {"100": {"p": 0.0, "tts99_us_secondary": math.inf}}, "spread": [1.0, math.inf], "n": 3}
    out = json.dumps(bench.finite(line), allow_nan=False)             # raises on inf / nan
    back = json.loads(out)
    assert back["tts99_us"] == {"primary": None, "secondary": None}
    assert back["tts99_by_budget"]["100"]["tts99_us_secondary"] is None
    assert back["spread"] == [1.0, None] and back["value"] == 1.5 and back["n"] == 3


def test_step_budgets_cover_the_metric_range():
    assert bench.BUDGETS[0] == 100 and bench.BUDGETS[-1] == 2000 and 1000 in bench.BUDGETS
