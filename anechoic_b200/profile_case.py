"""A small, fixed SCA workload for profiler captures (e.g. ncu --set full on one launch of one engine).

    python -m anechoic_b200.profile_case [--engine plain|tensor|cluster|auto] [--tensor-kind auto|int8|fp4]
                                         [--chains 148] [--steps 200] [--n 2000] [--torus L1xL2]
                                         [--sched counted|sparse51] [--launches 2] [--phases]

Runs --launches launches of --chains anneals over --steps steps, and prints the device time of each and the kernel
that ran. The instance is the N-spin +-1 complete graph (generator seed 20261004), or with --torus the +-1 toroidal
grid of the 51-instance sparse batch (seed 20261008 + 1000 L1 + L2, bias in [-2, 2]; 100x200 is its 20000-spin
member). Schedules:
- counted: counted Onsager, lambda 1.05, ramp, t0 30, t1 5, q 4;
- sparse51: the sparse batch's temperature-scaled correction, kappa 2, ramp, t0 6, t1 0.5, q 1.5.
--phases adds the tensor engine's per-phase cycle counters (SM cycles per step).
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
    ap.add_argument("--torus", default=None, help="L1xL2: the sparse batch's +-1 toroidal grid instead of K_n")
    ap.add_argument("--sched", default="counted", choices=["counted", "sparse51"])
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--tensor-kind", default="auto", choices=["auto", "int8", "fp4"])
    ap.add_argument("--phases", action="store_true")
    a = ap.parse_args()
    if a.torus:
        from .instances import torus
        l1, l2 = (int(v) for v in a.torus.lower().split("x"))
        inst = torus(l1, l2, 20261008 + l1 * 1000 + l2, True, 2)
    else:
        inst = A.complete_pm1(a.n, 20261004)
    dev = A.DeviceInstance(inst)
    if a.sched == "sparse51":
        tb = A.Tables.from_schedule(A.Schedule(S=a.steps, t0=6.0, t1=0.5, q=1.5, kappa=2.0, ramp=True))
    else:
        tb = A.Tables.from_schedule(A.Schedule(S=a.steps, lam=1.05, ramp=True))
    for k in range(a.launches):
        r = A.run(dev, tb, 20261004, k * a.chains, a.chains, engine=a.engine, tensor_kind=a.tensor_kind,
                  profile=a.phases and k == a.launches - 1)
        line = {"launch": k, "engine": a.engine, "kernel": r.kernel, "chains": a.chains, "steps": a.steps, "n": inst.n,
                "device_ms": r.device_ms, "mean_flips_per_step": float(r.flips.mean() / a.steps)}
        if r.profile:
            line["phases"] = {k2: round(v, 1) for k2, v in r.profile.items()}
        print(json.dumps(line))


if __name__ == "__main__":
    main()
