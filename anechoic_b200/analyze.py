"""TTS99 estimators over a cohort of runs, computed from the run files the CLI writes (PREFIX.summary.json and
PREFIX.batches.jsonl), with the reference's definitions (gpu/onsager_v2_20261007/src/analyze.py:15-88):

  primary    P_batch = fraction of batches with at least one success;  TTS99 = t ln 0.01 / ln(1 - P_batch)
             (= t when P_batch = 1, infinite when P_batch = 0)
  secondary  p = per-trial success fraction;  TTS99 = t ln 0.01 / (B ln(1 - p))  (0 when p = 1)
  whole      t * max(1, ceil(ln 0.01 / ln(1 - P_batch)))  (whole batches)
  t          mean device time of one launch (one batch of B anneals)
  intervals  Wilson score 95 % on P_batch and p, mapped through the monotone TTS formulas

    python -m anechoic_b200.analyze PREFIX.summary.json [...]     one JSON line per run
"""
from __future__ import annotations

import json
import math
import os
import sys

Z95 = 1.959963984540054     # two-sided 95 % normal quantile
LN01 = math.log(0.01)


def wilson(k: float, n: float):
    """Wilson score 95 % interval of a binomial proportion k / n, clipped to [0, 1]; (0, 1) when n = 0."""
    if n <= 0:
        return (0.0, 1.0)
    p = k / n
    z2 = Z95 * Z95
    den = 1.0 + z2 / n
    mid = (p + z2 / (2.0 * n)) / den
    rad = Z95 * math.sqrt(p * (1.0 - p) / n + z2 / (4.0 * n * n)) / den
    return (max(0.0, mid - rad), min(1.0, mid + rad))


def _log1m(P: float) -> float:
    """ln(1 - P), or None when it rounds to 0 (P within rounding of 0: the time to solution is then unbounded).
    The reference's estimators divide by it and raise ZeroDivisionError there (e.g. the Wilson lower bound of a
    cohort without successes); these return infinity instead."""
    v = math.log(1.0 - P)
    return v if v != 0.0 else None


def tts99(P: float, t: float) -> float:
    """Time to solution at 99 % from a per-batch success probability P and batch time t."""
    if P >= 1.0:
        return t
    if P <= 0.0:
        return math.inf
    d = _log1m(P)
    return math.inf if d is None else t * LN01 / d


def tts99_secondary(p: float, B: int, t: float) -> float:
    """Secondary TTS99 from the per-anneal success probability p with B anneals per batch, evaluated directly."""
    if p <= 0.0:
        return math.inf
    if p >= 1.0:
        return 0.0
    d = _log1m(p)
    return math.inf if d is None else t * LN01 / (B * d)


def tts99_whole(P: float, t: float) -> float:
    """TTS99 in whole batches: t times the number of batches needed for 99 %."""
    if P >= 1.0:
        return t
    if P <= 0.0:
        return math.inf
    d = _log1m(P)
    return math.inf if d is None else t * max(1, math.ceil(LN01 / d))


def load_run(prefix: str):
    with open(prefix + ".summary.json") as f:
        summary = json.load(f)
    with open(prefix + ".batches.jsonl") as f:
        batches = [json.loads(line) for line in f if line.strip()]
    return summary, batches


def estimate(prefix: str) -> dict:
    """Estimators of one run from its files: every field of the reference's estimate() under the same names
    (analyze.py:56-80), plus t1, engine, kernel and n."""
    s, bat = load_run(prefix)
    B, nb = int(s["chains"]), len(bat)
    t = sum(b["device_ms"] for b in bat) / nb
    host = sum(b["host_ms"] for b in bat) / nb
    kb = sum(1 for b in bat if b["successes"] > 0)
    kt = sum(int(b["successes"]) for b in bat)
    nt = B * nb
    Pb, p = kb / nb, kt / nt
    Pb_ci, p_ci = wilson(kb, nb), wilson(kt, nt)
    out = {k: s.get(k) for k in ("cs", "groups", "steps", "t0", "t1", "q", "ramp", "tec_jv", "trial_offset",
                                  "engine", "kernel", "n", "gpu_before", "gpu_after")}
    out.update(lam=s.get("lambda"), kappa=s.get("tecT_kappa"))      # the reference's estimate() names
    out.update({"lambda": s.get("lambda"), "tecT_kappa": s.get("tecT_kappa")})   # the run files' names
    out.update(prefix=os.path.basename(prefix), B=B, batches=nb, successes=kt, trials=nt, p=p, p_wilson95=list(p_ci),
               batches_with_success=kb, P_batch=Pb, P_batch_wilson95=list(Pb_ci), t_batch_ms=t,
               t_batch_min_ms=min(b["device_ms"] for b in bat), t_batch_max_ms=max(b["device_ms"] for b in bat),
               host_ms=host, us_per_step=1000.0 * t / s["steps"],
               tts_primary_ms=tts99(Pb, t), tts_primary_ci_ms=[tts99(Pb_ci[1], t), tts99(Pb_ci[0], t)],
               tts_primary_whole_ms=tts99_whole(Pb, t),
               tts_secondary_ms=tts99_secondary(p, B, t),
               tts_secondary_ci_ms=[tts99_secondary(p_ci[1], B, t), tts99_secondary(p_ci[0], B, t)],
               cut_mismatches=s.get("cut_mismatches"))
    return out


def selection_score(e: dict, which: str = "primary") -> float:
    """Pilot selection score: TTS99 at the Wilson 95 % lower bound of P_batch (primary) or p (secondary)."""
    if which == "primary":
        return tts99(e["P_batch_wilson95"][0], e["t_batch_ms"])
    return tts99_secondary(e["p_wilson95"][0], e["B"], e["t_batch_ms"])


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    for path in sorted(argv):
        if path.endswith(".summary.json"):
            print(json.dumps(estimate(path[: -len(".summary.json")])))
    return 0


if __name__ == "__main__":
    sys.exit(main())
