"""Generate tests/golden/float_agreement.json from the REFERENCE's float research model of the engine.

research/optimum_mitigation_20261007/sca_fast.py::run_cfg (numba) runs the same clipped synchronous SCA as the exact
engine, with float64 thresholds and its own RNG (sca_fast.py:1-20). It is imported from the reference tree (this
container only) and run on the synthetic N = 2000 +-1 instance (seed 20261004) for three matched schedules. For each
schedule, 4096 trials record the number of final cuts at or above three targets: the float model's own quartiles.
The exact engine's GPU test (tests/test_float_agreement.py) compares its success proportions with these counts
(two-proportion z-test), as the reference compares its exact and float models
(gpu/multibit_bias_20261008/REPORT.md:62). Run from the repository root with the reference project's root:

    python tests/golden/make_float_agreement.py --ref-root REFERENCE_ROOT
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
MODEL_DIR = "research/optimum_mitigation_20261007"     # the float model's directory within the reference project
sys.path.insert(0, ROOT)

from anechoic_b200 import instances as I  # noqa: E402

# (mode, exact-engine Schedule kwargs, float-model cfg)
CASES = [
    ("onsager", dict(S=300, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True),
     dict(family="onsager", S=300, T0=30.0, T1=5.0, q=4.0, lam=1.05, ramp=True)),
    ("tecT", dict(S=280, t0=15.0, t1=5.0, q=8.0, kappa=2.0, ramp=True),
     dict(family="tecT", S=280, T0=15.0, T1=5.0, q=8.0, kappa=2.0, ramp=True)),
    ("plain", dict(S=300, t0=30.0, t1=5.0, q=4.0),
     dict(family="plain", S=300, T0=30.0, T1=5.0, q=4.0)),
]
B = 4096


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", required=True, help="root directory of the reference project")
    a = ap.parse_args(argv)
    sys.path.insert(0, os.path.join(a.ref_root, MODEL_DIR))
    import sca_fast as F
    inst = I.complete_pm1(2000, 20261004)
    J = inst.dense.astype(np.float32)
    J2 = (2 * inst.dense).astype(np.int8)
    sumw = float(inst.stats()["sumw"])
    out = []
    for k, (mode, sched, cfg) in enumerate(CASES):
        cut = F.run_cfg(J, J2, sumw, cfg, B, 1000 + k)["cut"]
        targets = [int(np.quantile(cut, p)) for p in (0.25, 0.5, 0.75)]
        out.append(dict(mode=mode, schedule=sched, float_cfg=cfg, trials=B, targets=targets,
                        successes=[int((cut >= t).sum()) for t in targets], mean_cut=float(cut.mean()),
                        std_cut=float(cut.std())))
        print(out[-1])
    with open(os.path.join(HERE, "float_agreement.json"), "w") as f:
        json.dump(dict(instance="complete_pm1(2000, 20261004)", model=MODEL_DIR + "/sca_fast.py::run_cfg", cases=out), f, indent=1)


if __name__ == "__main__":
    main()
