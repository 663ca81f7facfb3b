"""Exact engine vs the reference's float research model of the same dynamics (research/optimum_mitigation_20261007/
sca_fast.py::run_cfg: float64 thresholds, its own RNG). Its success counts at three targets per schedule on the
synthetic N = 2000 +-1 instance are committed in tests/golden/float_agreement.json (tests/golden/
make_float_agreement.py). The engine runs the same schedules on 4096 anneals here. The proportions of cuts at or
above each target must agree by a two-proportion z-test (|z| < 4), and the mean cuts within 4 standard errors, as
the reference checks its exact engine against its float models (gpu/multibit_bias_20261008/REPORT.md:62)."""
import json
import math
import os

import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I

pytestmark = pytest.mark.gpu
FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "float_agreement.json")


def _z(k1, n1, k2, n2):
    p = (k1 + k2) / (n1 + n2)
    return (k2 / n2 - k1 / n1) / math.sqrt(p * (1 - p) * (1 / n1 + 1 / n2))


def test_success_proportions_agree(cuda):
    with open(FIX) as f:
        d = json.load(f)
    inst = I.complete_pm1(2000, 20261004)
    dev = A.DeviceInstance(inst)
    sumw = dev.info["sumw"]
    n = 4096
    for c in d["cases"]:
        r = A.run(dev, A.Tables.from_schedule(A.Schedule(**c["schedule"])), 20261004, 8_000_000, n)
        cut = r.cuts(sumw)
        for t, k in zip(c["targets"], c["successes"]):
            z = _z(k, c["trials"], int((cut >= t).sum()), n)
            assert abs(z) < 4, (c["mode"], t, z)
        se = math.sqrt(c["std_cut"] ** 2 / c["trials"] + float(np.var(cut)) / n)
        assert abs(float(cut.mean()) - c["mean_cut"]) < 4 * se, (c["mode"], float(cut.mean()), c["mean_cut"])
