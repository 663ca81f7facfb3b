"""Generate tests/golden/analyze_estimates.json: the reference's own TTS99 estimators run on run files in this
project's CLI format.

Each case is a cohort of batches (anneals per batch, per-batch successes, device and host times). Its
PREFIX.summary.json is built by the CLI's own record builder (anechoic_b200.cli.make_summary) and its
PREFIX.batches.jsonl in the CLI's batch-line format; the reference's estimate() and selection_score()
(gpu/onsager_v2_20261007/src/analyze.py:56-88, imported from the reference tree given on the command line) read
them unchanged. The fixture stores the two files' text and the reference's outputs (or the exception it raises);
tests/test_analyze.py writes the files back and requires anechoic_b200.analyze to give the same values. Run from the repository root:

    python tests/golden/make_analyze_golden.py --ref-root REFERENCE_ROOT
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

ANALYZE = "gpu/onsager_v2_20261007/src/analyze.py"   # within the reference project

# (name, anneals per batch, per-batch successes, per-batch device ms)
CASES = [
    ("mixed", 1024, [0, 3, 1, 0, 7, 0, 0, 2], [9.0, 9.1, 8.9, 9.05, 9.2, 8.95, 9.0, 9.1]),
    ("every_batch", 240, [5, 1, 9, 2], [1.5, 1.6, 1.55, 1.52]),
    ("none", 120, [0, 0, 0], [0.8, 0.81, 0.79]),
    ("every_trial", 16, [16, 16], [2.0, 2.2]),
    ("one_batch", 64, [1], [3.0]),
    ("rare", 4096, [0] * 19 + [1], [36.0 + 0.01 * k for k in range(20)]),
]


def enc(v):
    """JSON-safe form of an estimator output (inf as a string)."""
    if isinstance(v, float) and not math.isfinite(v):
        return "inf" if v > 0 else "-inf"
    if isinstance(v, (list, tuple)):
        return [enc(x) for x in v]
    return v


def run_files(name, B, succ, dms):
    """The summary.json and batches.jsonl text the CLI writes for this cohort."""
    from anechoic_b200 import cli
    from anechoic_b200.engine import Schedule
    sc = Schedule(S=1000, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True)
    o = dict(chains=B, batches=len(succ), geometry={}, engine="auto", tensor_kind="auto", warmup=1, seed=20261004,
             offset=0, trace=0)
    hms = [d + 0.25 for d in dms]
    bsucc = sum(1 for s in succ if s > 0)
    summary = cli.make_summary(o, sc, 2000, "tensor-fp4", sum(succ), bsucc, dms, hms, 0, None, 32720, None, "?")
    summary["device"], summary["uuid"], summary["gpu_after"] = "synthetic", "", "?"
    batches = "".join(json.dumps(dict(batch=b, chains=B, trial_offset=b * B, device_ms=dms[b], host_ms=hms[b],
                                      successes=succ[b]), separators=(",", ":")) + "\n" for b in range(len(succ)))
    return json.dumps(summary) + "\n", batches


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", required=True, help="root directory of the reference project")
    a = ap.parse_args(argv)
    spec = importlib.util.spec_from_file_location("ref_analyze", os.path.join(a.ref_root, ANALYZE))
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    out = []
    with tempfile.TemporaryDirectory() as d:
        for name, B, succ, dms in CASES:
            summary, batches = run_files(name, B, succ, dms)
            prefix = os.path.join(d, name)
            with open(prefix + ".summary.json", "w") as f:
                f.write(summary)
            with open(prefix + ".batches.jsonl", "w") as f:
                f.write(batches)
            try:
                e = ref.estimate(prefix)
                e["selection_primary"] = ref.selection_score(e, "primary")
                e["selection_secondary"] = ref.selection_score(e, "secondary")
            except ArithmeticError as ex:
                # the reference's estimator raises here (a Wilson bound within rounding of 0 reaches log(1 - P) = 0)
                out.append(dict(name=name, summary=summary, batches=batches, raises=type(ex).__name__))
                print(name, "raises", type(ex).__name__)
                continue
            out.append(dict(name=name, summary=summary, batches=batches, expected={k: enc(v) for k, v in e.items()}))
            print(name, e["tts_primary_ms"], e["tts_secondary_ms"])
    with open(os.path.join(HERE, "analyze_estimates.json"), "w") as f:
        json.dump(dict(estimator=ANALYZE + " estimate() / selection_score()", cases=out), f, indent=1)


if __name__ == "__main__":
    main()
