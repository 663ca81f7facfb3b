"""A small, fixed SCA workload for profiler captures (e.g. ncu --set full on one launch of one engine).

    python -m anechoic_b200.profile_case [--engine plain|tensor] [--tensor-kind auto|int8|fp4] [--chains 148]
                                         [--steps 200] [--n 2000] [--launches 2] [--phases]

Runs --launches launches of --chains anneals of the N-spin +-1 complete graph (generator seed 20261004) with the
counted Onsager schedule (lambda 1.05, ramp, t0 30, t1 5, q 4) over --steps steps, and prints the device time of each
and the kernel that ran. --phases adds the tensor engine's per-phase cycle counters (SM cycles per step).
"""
from __future__ import annotations

import argparse
import json

import anechoic_b200 as A


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--engine", default="plain", choices=["auto", "plain", "tensor", "cluster"])
    ap.add_argument("--chains", type=int, default=148)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--tensor-kind", default="auto", choices=["auto", "int8", "fp4"])
    ap.add_argument("--phases", action="store_true")
    a = ap.parse_args()
    inst = A.complete_pm1(a.n, 20261004)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(S=a.steps, lam=1.05, ramp=True))
    for k in range(a.launches):
        r = A.run(dev, tb, 20261004, k * a.chains, a.chains, engine=a.engine, tensor_kind=a.tensor_kind,
                  profile=a.phases and k == a.launches - 1)
        line = {"launch": k, "engine": a.engine, "kernel": r.kernel, "chains": a.chains, "steps": a.steps, "n": a.n,
                "device_ms": r.device_ms, "mean_flips_per_step": float(r.flips.mean() / a.steps)}
        if r.profile:
            line["phases"] = {k2: round(v, 1) for k2, v in r.profile.items()}
        print(json.dumps(line))


if __name__ == "__main__":
    main()
