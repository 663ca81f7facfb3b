"""Generate tests/golden/sparse_tuning_b200.json on a B200: the CSR-pass tuner's probe times against full-run times.

For each sparse instance class of the 51-instance batch (toroidal grid, degree-6 and degree-12 random graphs, the
dense Erdos-Renyi class), the plain engine's first synchronous run makes the tuner probe each compiled variant
(anc_sparse_tuning: the first min(S, 64) steps of up to one wave of anneals, the second of two launches timed); each
variant then runs the full schedule (S = 1000, one wave of 148 anneals, the variant forced through the options) for
its device time. tests/test_autotune.py checks on this record that the probe's pick is within 5 % of the fastest
variant on the full run. Run on a GPU box from the repository root:

    python tests/golden/make_sparse_tuning.py
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import anechoic_b200 as A  # noqa: E402
from anechoic_b200 import _lib  # noqa: E402
from anechoic_b200 import instances as I  # noqa: E402

SCHED = dict(S=1000, t0=6.0, t1=0.5, q=1.5, kappa=2.0, ramp=True)
CASES = [
    ("torus_100x200", lambda: I.torus(100, 200, 20261008 + 100 * 1000 + 200, True, 2)),
    ("torus_40x50", lambda: I.torus(40, 50, 20261008 + 40 * 1000 + 50, True, 2)),
    ("deg6_n5000", lambda: I.random_graph(5000, 15000, True, 20261408, 2)),
    ("deg6_n2000", lambda: I.random_graph(2000, 6000, False, 20261409, 2)),
    ("deg12_n2000", lambda: I.random_graph(2000, 11778, True, 20261308, 2)),
    ("er_n800", lambda: I.random_graph(800, 19176, True, 20261013, 2)),
    ("er_n2000", lambda: I.random_graph(2000, 19990, False, 20261208, 2)),
]
ANNEALS = 148


def main():
    L = _lib.load()
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    out = []
    for name, build in CASES:
        inst = build()
        dev = A.DeviceInstance(inst)
        A.run(dev, tb, 7, 0, ANNEALS, engine="plain")          # the first synchronous run tunes
        v = C.c_int()
        us = (C.c_double * 4)()
        _lib.check(L.anc_sparse_tuning(dev._h, C.byref(v), us))
        full = []
        for forced in range(1, 5):
            o = _lib.opts("plain")
            o.sparse_variant = forced
            ms = []
            for rep in range(3):
                W = A.spin_words(inst.n)
                sp = np.zeros((ANNEALS, W), np.uint64)
                sh, bs, fl = (np.zeros(ANNEALS, np.int64) for _ in range(3))
                _lib.check(L.anc_run(dev._h, tb._h, 7, 1000 * (rep + 1), ANNEALS, C.byref(o), sp.ctypes.data,
                                     sh.ctypes.data, bs.ctypes.data, fl.ctypes.data, None))
                ms.append(L.anc_last_device_ms())
            full.append(min(ms[1:]))
        rec = dict(instance=name, n=inst.n, edges=int(len(inst.col) // 2), picked=v.value,
                   probe_us_per_step=[us[k] for k in range(4)], full_ms=full)
        print(json.dumps(rec))
        out.append(rec)
    with open(os.path.join(HERE, "sparse_tuning_b200.json"), "w") as f:
        json.dump(dict(schedule=SCHED, anneals=ANNEALS, variants=[[1, 8], [1, 4], [2, 4], [1, 16]], cases=out), f,
                  indent=1)


if __name__ == "__main__":
    main()
