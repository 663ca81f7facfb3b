"""Measures the device time of each engine on a grid of instances, schedules and batch sizes (run on a B200):

    python tests/golden/make_engine_times.py > tests/golden/engine_times_b200.json

Per case: the instance (n, kbits), the schedule, the anneals per launch, each engine's device time (ms, the least of
three launches on fresh trial ids after a warm-up launch), the flip fraction seen (flips per spin per step), the
anneals per wave of each engine and what engine="auto" picks once it has seen that flip fraction.
tests/test_autoselect.py checks the cost model against these times on the CPU.
"""
import json
import sys

import anechoic_b200 as A
from anechoic_b200 import instances as I

SCHEDULES = {"default": dict(S=1000, lam=1.05, ramp=True),
             "tect": dict(S=120, t0=15.0, q=8.0, kappa=2.0, ramp=True),
             "cold": dict(S=300, t0=4.0, t1=1.0, q=4.0, lam=1.05, ramp=True)}
CHAINS = (1, 16, 32, 64, 148, 200, 296)


def cases():
    for n in (500, 1000, 1500, 2000, 3000, 4000, 10000):
        yield f"pm1_{n}", I.complete_pm1(n, 20261004), ("default", "tect", "cold") if n in (500, 2000) else (
            "default", "tect")
    for name, inst in (("k2_2000", I.random_kbit(2000, 2, 1, pzero=0.5)), ("k4_2000", I.random_kbit(2000, 4, 2)),
                       ("k3_1000", I.random_kbit(1000, 3, 3)), ("k4_3000", I.random_kbit(3000, 4, 4))):
        yield name, inst, ("default", "tect")


def main():
    rows = []
    for name, inst, scheds in cases():
        dev = A.DeviceInstance(inst)
        for sn in scheds:
            sc = SCHEDULES[sn]
            tb = A.Tables.from_schedule(A.Schedule(**sc))
            for c in CHAINS:
                row = {"case": name, "n": inst.n, "kbits": dev.info["kbits"], "sched": sn, "S": sc["S"], "chains": c,
                       "ms": {}, "kernel": {}}
                flips = None
                for e in ("plain", "cluster", "tensor"):
                    if e == "cluster" and (dev.info["kbits"] != 1 or inst.n > 2048):
                        continue
                    times = []
                    for k in range(4):
                        r = A.run(dev, tb, 7, k * c, c, engine=e)
                        times.append(r.device_ms)
                    row["ms"][e] = round(min(times[1:]), 4)
                    row["kernel"][e] = r.kernel
                    flips = r.flips
                row["flip_fraction"] = round(float(flips.mean()) / (inst.n * sc["S"]), 5)
                ch = A.auto_choice(dev, tb, c)
                row["per_wave"] = ch["per_wave"]
                row["fp4"] = row["kernel"].get("tensor") == "tensor-fp4"
                row["auto_pick"] = ch["pick"]
                rows.append(row)
                print(json.dumps(row), file=sys.stderr, flush=True)
    json.dump({"device": "B200", "cases": rows}, sys.stdout, indent=0)
    print()


if __name__ == "__main__":
    main()
