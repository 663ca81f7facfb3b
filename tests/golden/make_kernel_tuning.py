"""Generate tests/golden/kernel_tuning_b200.json on a B200: the dense-kernel tuner's probe times against full-run times.

Cases: dense instances on the plain engine (rows per batch: three variants for 1-bit couplings, two for 2-bit) and the
fp4 kernel (ring depth 4 / 6 / 5 / 3) at one and at eight replica groups. Tuning keys (device, kernel, NP, K, replica
groups) live for the process, so each case runs in a fresh process: its first synchronous run makes the library probe
every variant (anc_kernel_tuning: the first min(S, 256) steps, the least of two timed launches after one); then each variant,
forced through anc_run_opts.kernel_variant, runs the full schedule (the least of three launches after a warm-up).
tests/test_autotune.py checks on this record that the probe's pick is within 5 % of the fastest variant on the full
run. Run on a GPU box from the repository root:

    python tests/golden/make_kernel_tuning.py
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SCHEDULES = {"default": dict(S=1000, lam=1.05, ramp=True),
             "tect": dict(S=120, t0=15.0, q=8.0, kappa=2.0, ramp=True),
             "cold": dict(S=300, t0=4.0, t1=1.0, q=4.0, lam=1.05, ramp=True)}
# name, instance builder (instances module), schedule, engine, anneals
CASES = [
    ("pm1_500", "complete_pm1(500, 20261004)", "default", "plain", 148),
    ("pm1_500", "complete_pm1(500, 20261004)", "cold", "plain", 148),
    ("pm1_2000", "complete_pm1(2000, 20261004)", "default", "plain", 148),
    ("pm1_2000", "complete_pm1(2000, 20261004)", "tect", "plain", 148),
    ("pm1_4000", "complete_pm1(4000, 20261004)", "default", "plain", 148),
    ("pm1_10000", "complete_pm1(10000, 20261004)", "tect", "plain", 148),
    ("k2_2000", "random_kbit(2000, 2, 1, pzero=0.5)", "default", "plain", 148),
    ("k2_3000", "random_kbit(3000, 2, 7, pzero=0.3, bmax=4)", "tect", "plain", 148),
    ("pm1_2000", "complete_pm1(2000, 20261004)", "default", "fp4", 128),
    ("pm1_2000", "complete_pm1(2000, 20261004)", "default", "fp4", 1024),
    ("pm1_2000", "complete_pm1(2000, 20261004)", "tect", "fp4", 1024),
    ("k2_2000", "random_kbit(2000, 2, 1, pzero=0.5)", "default", "fp4", 1024),
]
KERNEL = {"plain": 1, "fp4": 3}


def one_case(idx: int) -> dict:
    import numpy as np
    import anechoic_b200 as A
    from anechoic_b200 import _lib
    from anechoic_b200 import instances as I
    name, build, sched, engine, nchains = CASES[idx]
    L = _lib.load()
    inst = eval("I." + build)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(**SCHEDULES[sched]))
    eng = "plain" if engine == "plain" else "tensor"
    kind = "fp4" if engine == "fp4" else "auto"
    A.run(dev, tb, 7, 0, nchains, engine=eng, tensor_kind=kind)          # the first synchronous run tunes
    v, nv = C.c_int(), C.c_int()
    us = (C.c_double * 4)()
    _lib.check(L.anc_kernel_tuning(dev._h, KERNEL[engine], nchains, C.byref(v), C.byref(nv), us))
    full = []
    for forced in range(1, nv.value + 1):
        o = _lib.opts(eng, tensor_kind=kind)
        o.kernel_variant = forced
        ms = []
        for rep in range(4):
            sp = np.zeros((nchains, A.spin_words(inst.n)), np.uint64)
            sh, bs, fl = (np.zeros(nchains, np.int64) for _ in range(3))
            _lib.check(L.anc_run(dev._h, tb._h, 7, 100000 * (rep + 1), nchains, C.byref(o), sp.ctypes.data,
                                 sh.ctypes.data, bs.ctypes.data, fl.ctypes.data, None))
            ms.append(L.anc_last_device_ms())
        full.append(round(min(ms[1:]), 4))
    return dict(instance=name, schedule=sched, kernel=engine, anneals=nchains, n=inst.n, kbits=dev.info["kbits"],
                picked=v.value, probe_us_per_step=[round(us[k], 4) for k in range(nv.value)], full_ms=full)


def main():
    if len(sys.argv) == 3 and sys.argv[1] == "--case":
        print(json.dumps(one_case(int(sys.argv[2]))))
        return
    out = []
    for k in range(len(CASES)):
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--case", str(k)], capture_output=True,
                           text=True, cwd=ROOT)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise SystemExit(f"case {k} failed")
        rec = json.loads(r.stdout.strip().splitlines()[-1])
        print(json.dumps(rec), flush=True)
        out.append(rec)
    with open(os.path.join(HERE, "kernel_tuning_b200.json"), "w") as f:
        json.dump(dict(schedules=SCHEDULES, variants={"plain_k1": ["8 rows + next 8 ahead", "8 rows", "16 rows"],
                                                      "plain_k2": ["8 rows", "16 rows"],
                                                      "fp4": ["4 stages", "6 stages", "5 stages", "3 stages"]},
                       cases=out), f, indent=1)


if __name__ == "__main__":
    main()
