"""Cohort driver: the reference's measurement protocol (gpu/onsager_v2_20261007/src/run_protocol.sh:1-132) run on
this project's engines through the drop-in CLI, which writes the reference's run files. The estimators are those
of anechoic_b200.analyze.

    python -m anechoic_b200.cohort PHASE --graph F --results DIR [--target CUT] [--seed S] [--scale X]
                                   [--batch-sizes 1,120,240,480]

Phases, run in the order V K M P H (W optional). Every run refuses to overwrite its outputs, and V must pass before
any other phase:
  V  validation: each engine that supports the instance runs the plain, counted-Onsager, TEC-T and TEC schedules
     with traces and --check-fields 1. Every returned cut and field is rescored on the host (0 mismatches), and the
     spin files of all engines must be byte-identical for the same (seed, trial ids, schedule). The reference
     validates its kernel variants against the golden model here; the golden model belongs to the tests in this
     project (tests/), so the driver cross-checks the engines and rescores on the host instead.
  K  engine selection: every engine that supports the instance, timed at each batch size on configuration X5;
     the fastest per batch size is recorded (results/K/selected_engines.json).
  M  the named configurations (CFG) at every batch size, on the selected engine.
  P  pilot: grid of modes x q x t0 x S at batch sizes 240 and 120 (32 batches each at --scale 1). Each cell's
     score is TTS99 at the Wilson 95 % lower bound of its success probability (primary: per batch; secondary: per
     anneal); the lowest score wins (results/P/selected_{primary,secondary}.json).
  H  held-out: the selected schedules again on fresh trial ids (128 batches at the selected size, 256 single
     anneals, 128 batches at the other size).
  W  power: back-to-back batches of the primary selection for --burn seconds while nvidia-smi samples power and
     clocks (read only).
--scale multiplies every batch count (at least 1 batch), so a short protocol keeps the same structure.
"""
from __future__ import annotations

import glob
import json
import os
import subprocess
import sys
import time
from typing import Dict, List

from . import analyze, cli

# the reference's named configurations (run_protocol.sh:11-19)
CFG = {
    "X5": "--q 8 --tecT 1.75 --ramp --t0 15 --steps 280",
    "X1": "--q 8 --tecT 1.75 --ramp --t0 15 --steps 320",
    "X4": "--q 8 --tecT 2.0 --ramp --t0 15 --steps 760",
    "X2": "--q 6 --lambda 0.9 --ramp --t0 15 --steps 320",
    "O1": "--q 8 --lambda 1.05 --ramp --t0 12 --steps 960",
    "O4": "--q 6 --lambda 0.9 --t0 12 --steps 360",
    "P4": "--q 8 --lambda 0 --t0 30 --steps 960",
}
ORDER = ["X5", "X1", "X4", "X2", "O1", "O4", "P4"]
# validation schedules (run_protocol.sh:32-33)
VSCHED = {
    "plain": "--q 4 --lambda 0 --t0 30 --steps 40",
    "onsager": "--q 8 --lambda 1.05 --ramp --t0 12 --steps 960",
    "tecT": "--q 8 --tecT 1.75 --ramp --t0 15 --steps 280",
    "tec": "--q 8 --tec-jv -4 --t0 30 --steps 100",
}
PILOT_MODES = ["--tecT 1.5", "--tecT 1.75", "--tecT 2.0", "--lambda 0.9", "--lambda 1.05"]
PILOT_Q = [6, 8]
PILOT_T0 = [12, 15]
PILOT_S = [80, 120, 160, 200, 240, 280]


class Ctx:
    def __init__(self, graph: str, results: str, target: int, seed: int, scale: float, sizes: List[int],
                 log=print):
        self.graph, self.results, self.target, self.seed, self.scale, self.sizes = graph, results, target, seed, scale, sizes
        self.log = log

    def nb(self, batches: int) -> int:
        return max(1, int(round(batches * self.scale)))

    def path(self, *p) -> str:
        return os.path.join(self.results, *p)

    def run(self, tag: str, chains: int, batches: int, offset: int, sched: str, engine: str = "auto",
            extra: List[str] = ()) -> Dict:
        """One CLI run writing results/<tag>.*; refuses to overwrite. Returns its summary."""
        prefix = self.path(tag)
        if os.path.exists(prefix + ".summary.json") or os.path.exists(prefix + ".trials.jsonl"):
            raise FileExistsError("refusing to overwrite " + prefix)
        os.makedirs(os.path.dirname(prefix), exist_ok=True)
        argv = ["--graph", self.graph, "--output", prefix, "--chains", str(chains), "--batches", str(batches),
                "--offset", str(offset), "--seed", str(self.seed), "--target", str(self.target), "--engine", engine,
                *sched.split(), *extra]
        rc = cli.main(argv)
        if rc == 1:
            raise RuntimeError(f"run {tag} failed")
        with open(prefix + ".summary.json") as f:
            s = json.load(f)
        s["_rc"] = rc
        self.log(json.dumps({"tag": tag, "engine": s["kernel"], "chains": chains, "batches": batches,
                             "device_ms_mean": s["device_ms_mean"], "p": s["p"], "rc": rc}))
        return s


def engines_for(graph: str) -> List[str]:
    """Engines that support the instance (the cluster engine: 1-bit couplings, n <= 2048; the tensor engine: dense,
    NP <= 4096)."""
    from . import instances
    from .engine import DeviceInstance
    inst = instances.load("graph", graph)
    info = DeviceInstance(inst).info
    out = ["plain"]
    if info["kbits"] == 1 and info["np"] == 2048:
        out.append("cluster")
    if not info["sparse"] and info["np"] <= 4096:
        out.append("tensor")
    return out


def _require(path: str, what: str):
    if not os.path.exists(path):
        raise RuntimeError(f"{what} missing ({path}): run the earlier phase first")


def _validated(ctx: Ctx):
    p = ctx.path("V", "validation_summary.json")
    _require(p, "validation")
    with open(p) as f:
        if json.load(f).get("verdict") != "PASS":
            raise RuntimeError("validation did not pass")


def _engine(ctx: Ctx, B: int) -> str:
    p = ctx.path("K", "selected_engines.json")
    _require(p, "engine selection")
    with open(p) as f:
        sel = json.load(f)
    return sel.get(str(B)) or sel[max(sel, key=lambda k: int(k))]


def phase_V(ctx: Ctx):
    engines = engines_for(ctx.graph)
    rows, ok = [], True
    cases = [(m, c, off) for m in VSCHED for c, off in ((4, 900000), (8, 31337))]
    for mode, chains, off in cases:
        spins = {}
        for e in engines:
            tag = f"V/{mode}_{e}_b{chains}"
            s = ctx.run(tag, chains, 1, off, VSCHED[mode], engine=e, extra=["--trace", "1", "--check-fields", "1"])
            good = s["_rc"] == 0 and s["cut_mismatches"] == 0 and not s.get("field_mismatches")
            with open(ctx.path(tag) + ".spins.bin", "rb") as f:
                spins[e] = f.read()
            rows.append(dict(tag=tag, engine=s["kernel"], trials=chains, host_rescoring_ok=good))
            ok &= good
        same = len(set(spins.values())) == 1
        rows.append(dict(mode=mode, chains=chains, offset=off, engines=engines, spins_identical=same))
        ok &= same
    verdict = "PASS" if ok else "FAIL"
    with open(ctx.path("V", "validation_summary.json"), "w") as f:
        json.dump(dict(verdict=verdict, engines=engines, rows=rows), f, indent=1)
    ctx.log("VALIDATION " + verdict)
    if not ok:
        raise RuntimeError("validation failed")


def phase_K(ctx: Ctx):
    _validated(ctx)
    engines = engines_for(ctx.graph)
    sel, times = {}, {}
    for i, B in enumerate(ctx.sizes):
        t = {}
        for j, e in enumerate(engines):
            s = ctx.run(f"K/b{B}_{e}", B, ctx.nb(16), 5000000 + 10000 * (4 * i + j), CFG["X5"], engine=e)
            t[e] = s["device_ms_mean"]
        sel[str(B)] = min(t, key=t.get)
        times[str(B)] = t
    with open(ctx.path("K", "selected_engines.json"), "w") as f:
        json.dump(sel, f, indent=1)
    with open(ctx.path("K", "times.json"), "w") as f:
        json.dump(times, f, indent=1)
    ctx.log(json.dumps({"selected": sel}))


def phase_M(ctx: Ctx):
    _validated(ctx)
    nbs = {1: 256, 120: 128, 240: 128, 480: 64}
    for i, c in enumerate(ORDER):
        base = 10000000 + i * 1000000
        for j, B in enumerate(ctx.sizes):
            ctx.run(f"M/{c}_b{B}", B, ctx.nb(nbs.get(B, 64)), base + 100000 * j, CFG[c], engine=_engine(ctx, B))


def pilot_cells():
    idx = 0
    for mode in PILOT_MODES:
        for q in PILOT_Q:
            for t0 in PILOT_T0:
                for S in PILOT_S:
                    yield idx, f"{mode} --ramp --q {q} --t0 {t0} --steps {S}"
                    idx += 1


def select_pilot(cells: List[Dict]) -> Dict[str, Dict]:
    """The lowest selection score per estimator (ties: the lower point estimate), as the reference's phase P."""
    out = {}
    for w in ("primary", "secondary"):
        for c in cells:
            c["score_" + w] = analyze.selection_score(c, w)
        out[w] = min(cells, key=lambda c: (c["score_" + w], c["tts_" + w + "_ms"]))
    return out


def phase_P(ctx: Ctx, grid=None):
    _validated(ctx)
    index = []
    for idx, args in (grid if grid is not None else pilot_cells()):
        base = 3000000 + idx * 8000
        for B in (240, 120):
            ctx.run(f"P/p{idx:03d}_b{B}", B, ctx.nb(32), base, args, engine=_engine(ctx, B))
        index.append(f"p{idx:03d} {args}")
    with open(ctx.path("P", "index.txt"), "w") as f:
        f.write("\n".join(index) + "\n")
    cells = [analyze.estimate(p[: -len(".summary.json")]) for p in sorted(glob.glob(ctx.path("P", "p*_b*.summary.json")))]
    best = select_pilot(cells)
    for w, c in best.items():
        with open(ctx.path("P", f"selected_{w}.json"), "w") as f:
            json.dump(c, f, indent=1)
        ctx.log(json.dumps({w: c["prefix"], "score": c["score_" + w], "tts_ms": c["tts_" + w + "_ms"]}))
    with open(ctx.path("P", "pilot_cells.json"), "w") as f:
        json.dump(cells, f, indent=0)


def _selected_args(ctx: Ctx, which: str):
    p = ctx.path("P", f"selected_{which}.json")
    _require(p, "pilot selection")
    with open(p) as f:
        c = json.load(f)
    mode = f"--tecT {c['tecT_kappa']:g}" if c["tecT_kappa"] > 0 else f"--lambda {c['lambda']:g}"
    return f"{mode} --ramp --q {c['q']:g} --t0 {c['t0']:g} --steps {c['steps']}", int(c["B"])


def phase_H(ctx: Ctx):
    _validated(ctx)
    a1, b1 = _selected_args(ctx, "primary")
    a2, b2 = _selected_args(ctx, "secondary")
    os.makedirs(ctx.path("H"), exist_ok=True)
    with open(ctx.path("H", "selected.txt"), "w") as f:
        f.write(f"primary: {a1} B={b1} ; secondary: {a2} B={b2}\n")
    ctx.run(f"H/primary_b{b1}", b1, ctx.nb(128), 4000000, a1, engine=_engine(ctx, b1))
    ctx.run("H/primary_b1", 1, ctx.nb(256), 4100000, a1, engine=_engine(ctx, 1))
    ob = 240 if b1 == 120 else 120
    ctx.run(f"H/primary_b{ob}", ob, ctx.nb(128), 4200000, a1, engine=_engine(ctx, ob))
    if (a2, b2) != (a1, b1):
        ctx.run(f"H/secondary_b{b2}", b2, ctx.nb(128), 4500000, a2, engine=_engine(ctx, b2))
    for p in sorted(glob.glob(ctx.path("H", "*.summary.json"))):
        ctx.log(json.dumps(analyze.estimate(p[: -len(".summary.json")])))


def phase_W(ctx: Ctx, burn_s: float = 75.0):
    """Back-to-back batches of the primary selection while nvidia-smi (if present) samples power and clocks."""
    _validated(ctx)
    a1, b1 = _selected_args(ctx, "primary")
    os.makedirs(ctx.path("W"), exist_ok=True)
    samples = ctx.path("W", "power_samples.csv")
    if os.path.exists(samples):
        raise FileExistsError("refusing to overwrite " + samples)
    smi = None
    try:
        smi = subprocess.Popen(["nvidia-smi", "--query-gpu=timestamp,utilization.gpu,memory.used,power.draw,clocks.sm",
                                "--format=csv,noheader", "-lms", "200"], stdout=open(samples, "w"),
                               stderr=subprocess.DEVNULL)
    except OSError:
        smi = None
    t0 = time.time()
    nb, dev_ms = 0, 0.0
    try:
        while time.time() - t0 < burn_s:
            tag = f"W/burn_{nb:05d}"
            s = ctx.run(tag, b1, 1, 6000000 + nb * b1, a1, engine=_engine(ctx, b1))
            dev_ms += s["device_ms_mean"]
            nb += 1
    finally:
        if smi is not None:
            smi.terminate()
            smi.wait(timeout=10)
    with open(ctx.path("W", "burn.json"), "w") as f:
        json.dump(dict(burn_seconds_wall=time.time() - t0, batches=nb, chains=b1, device_ms_per_batch=dev_ms / max(1, nb)),
                  f)


PHASES = {"V": phase_V, "K": phase_K, "M": phase_M, "P": phase_P, "H": phase_H, "W": phase_W}


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] not in PHASES:
        print("usage: python -m anechoic_b200.cohort V|K|M|P|H|W --graph F --results DIR [--target CUT] [--seed S] "
              "[--scale X] [--batch-sizes 1,120,240,480] [--burn SECONDS]", file=sys.stderr)
        return 1
    o = dict(graph=None, results="results", target=33000, seed=20261004, scale=1.0, sizes="1,120,240,480", burn=75.0)
    conv = dict(graph=str, results=str, target=int, seed=int, scale=float, sizes=str, burn=float)
    a = 1
    try:
        while a < len(argv):
            k = argv[a][2:].replace("batch-sizes", "sizes")
            if not argv[a].startswith("--") or k not in conv or a + 1 >= len(argv):
                raise ValueError("bad argument " + argv[a])
            o[k] = conv[k](argv[a + 1])
            a += 2
        if not o["graph"]:
            raise ValueError("--graph required")
        ctx = Ctx(o["graph"], o["results"], o["target"], o["seed"], o["scale"], [int(x) for x in o["sizes"].split(",")])
        if argv[0] == "W":
            phase_W(ctx, o["burn"])
        else:
            PHASES[argv[0]](ctx)
        return 0
    except (ValueError, RuntimeError, OSError) as e:
        print("FAIL: " + str(e), file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
