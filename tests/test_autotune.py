"""CPU: the run-time choices made from measurements hold up on the recorded B200 fixtures.

- The CSR-pass tuner (anc_api.cu tune_sparse) picks the variant with the least probe time (the first min(S, 64)
  steps of one wave). tests/golden/sparse_tuning_b200.json (tests/golden/make_sparse_tuning.py) records, per sparse
  instance class, each variant's probe time and its full-run time (S = 1000, 148 anneals): the probe's pick must be
  within 5 % of the fastest variant on the full run.
- The dense-kernel tuner (anc_api.cu tune_kernel) does the same for the plain engine's rows per batch on dense
  instances and the fp4 kernel's ring depth. tests/golden/kernel_tuning_b200.json (tests/golden/make_kernel_tuning.py)
  records, per instance, schedule and kernel, the library's pick and probe times and each variant's full-run time.
"""
import json
import os

import pytest

from tests.conftest import GOLDEN

FIXTURE = os.path.join(GOLDEN, "sparse_tuning_b200.json")


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="fixture not recorded yet")
def test_sparse_probe_pick_within_5_percent_of_best_full_run():
    with open(FIXTURE) as f:
        d = json.load(f)
    assert len(d["cases"]) >= 5 and len(d["variants"]) == 4
    for c in d["cases"]:
        probe, full = c["probe_us_per_step"], c["full_ms"]
        pick = min(range(4), key=lambda v: probe[v])
        assert c["picked"] == pick, c["instance"]            # the library kept the least probe time
        assert full[pick] <= 1.05 * min(full), (c["instance"], pick, full)


KFIXTURE = os.path.join(GOLDEN, "kernel_tuning_b200.json")


@pytest.mark.skipif(not os.path.exists(KFIXTURE), reason="fixture not recorded yet")
def test_dense_kernel_probe_pick_within_5_percent_of_best_full_run():
    with open(KFIXTURE) as f:
        d = json.load(f)
    kinds = {(c["kernel"], c["kbits"]) for c in d["cases"]}
    assert {("plain", 1), ("plain", 2), ("fp4", 1)} <= kinds and len(d["cases"]) >= 10
    for c in d["cases"]:
        probe, full = c["probe_us_per_step"], c["full_ms"]
        nv = len(full)
        assert nv == (4 if c["kernel"] == "fp4" else 3 if c["kbits"] == 1 else 2) and len(probe) == nv
        best = min(range(nv), key=lambda v: probe[v])
        pick = best if probe[best] < 0.99 * probe[0] else 0   # variant 0 unless another probes > 1 % faster
        ctx = (c["instance"], c["schedule"], c["kernel"], c["anneals"])
        assert c["picked"] == pick, ctx
        assert full[pick] <= 1.05 * min(full), (ctx, pick, full)
