#!/usr/bin/env python3
"""Benchmark of the SCA anneal path on B200: anneals/s and TTS99 to the target cut, one JSON line (rank 0).

Workload (one "step" = one batch): the N = 2000 +-1 complete graph (J_xy = J_yx iid uniform +-1, generator seed
20261004), 1024 concurrent anneals per GPU (trial ids rank*2^20 + step*1024 + c), counted Onsager correction
lambda = 1.05 with ramp, reference default schedule t0 = 30, t1 = 5, q = 4, S = 1000 steps, seed 20261004.
Target cut: 0.995 x the best cut of 1000 long anneals (S = 5000, same correction) of the same instance, run on the
exact engine outside the timed region. TTS99: primary t_batch ln(0.01)/ln(1 - P_batch), secondary
t_batch ln(0.01)/(B ln(1 - p)) (reference estimators, gpu/onsager_v2_20261007/src/analyze.py:15-47).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--engine auto|plain|tensor] [--impl ours|reference]

--impl reference times the reference's own CPU golden model (sca::run_trial_bias compiled unmodified into
oracle/_ref/libscaref.so) on all host threads over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SPINS = 2000
INSTANCE_SEED = 20261004
RUN_SEED = 20261004
CHAINS = 1024
SCHED = dict(S=1000, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True)
TARGET_SCHED = dict(S=5000, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True)
TARGET_ANNEALS = 1000
METRIC = "TTS99 (µs) to target cut and anneals/sec, batched vs plain engine, 1 B200"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1])); mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def profile_traffic(kernel: str):
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    e = d.get(kernel)
    return e.get("bytes_per_launch") if e else None


def tts99(P: float, t: float) -> float:
    if P >= 1.0:
        return t
    if P <= 0.0:
        return math.inf
    return t * math.log(0.01) / math.log(1.0 - P)


def tts99_secondary(p: float, B: int, t: float) -> float:
    if p <= 0.0:
        return math.inf
    if p >= 1.0:
        return 0.0
    return t * math.log(0.01) / (B * math.log(1.0 - p))


# ------------------------------------------------------------------------------------------------------ reference arm
def bench_reference(args, ws, rank):
    import numpy as np
    from anechoic_b200 import instances as I
    from oracle.oracle import Reference, REF_LIB
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libscaref.so was not built (reference "
                                                                "tree absent at build time)"}))
        return 0
    R = Reference()
    inst = I.complete_pm1(N_SPINS, INSTANCE_SEED)
    tb = R.build_tables(**SCHED)
    sample = max(cores, 8)     # anneals per step: one per host thread (bounded sample of the 1024-anneal batch)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        R.run_batch_bias(N_SPINS, inst.dense, None, tb, RUN_SEED, it * sample, sample, trace=False, threads=cores)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    per_step = sum(times) / len(times)
    value = sample / per_step
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "anneals/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"N={N_SPINS} +-1 complete graph, {CHAINS} anneals x S={SCHED['S']} counted Onsager "
                                   f"(lambda 1.05, ramp); reference CPU golden model on a {sample}-anneal sample",
                       "n": N_SPINS, "anneals": CHAINS, "S": SCHED["S"], "sample_anneals": sample},
            "cpu_baseline": {"value": value, "unit": "anneals/s", "cores": cores, "kind": "reference",
                             "sample": f"{sample} anneals x {SCHED['S']} steps per step on {cores} threads"},
            "e2e": {"value": value, "unit": "anneals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline_sample(budget_s: float = 15.0):
    """The reference's CPU golden model on the host cores (rank 0, N = 1 only): anneals/s on a bounded sample."""
    from anechoic_b200 import instances as I
    from oracle.oracle import Reference, REF_LIB, Restatement
    cores = os.cpu_count() or 1
    inst = I.complete_pm1(N_SPINS, INSTANCE_SEED)
    if os.path.exists(REF_LIB):
        R, kind = Reference(), "reference"
        tb = R.build_tables(**SCHED)
        run = lambda k, off: R.run_batch_bias(N_SPINS, inst.dense, None, tb, RUN_SEED, off, k, threads=cores)
    else:
        R, kind = Restatement(), "port"
        tb = R.tables(**SCHED)
        run = lambda k, off: R.run_batch(N_SPINS, tb, RUN_SEED, off, k, dense=inst.dense, trace=False, threads=cores)
    t0 = time.perf_counter(); run(cores, 0); first = time.perf_counter() - t0
    reps = max(1, int(budget_s / max(first, 1e-3)))
    t0 = time.perf_counter()
    for r in range(reps):
        run(cores, (r + 1) * cores)
    dt = time.perf_counter() - t0
    return {"value": reps * cores / dt, "unit": "anneals/s", "cores": cores, "kind": kind,
            "sample": f"{reps * cores} anneals (N={N_SPINS}, S={SCHED['S']}, counted Onsager) on {cores} threads, "
                      f"{dt:.1f} s"}


# ------------------------------------------------------------------------------------------------------ our arm
def bench_ours(args, ws, rank, local):
    import numpy as np
    import torch
    import anechoic_b200 as A
    from anechoic_b200 import _lib

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev_index = local
    inst = A.complete_pm1(N_SPINS, INSTANCE_SEED)
    dev = A.DeviceInstance(inst)
    sumw = dev.info["sumw"]
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    engine = args.engine

    # target cut (outside the timed region): best of 1000 long anneals on the exact engine
    ttb = A.Tables.from_schedule(A.Schedule(**TARGET_SCHED))
    tr = A.run(dev, ttb, RUN_SEED, 0xE0000000, TARGET_ANNEALS, engine=engine)
    best = int(tr.cuts(sumw).max())
    target = math.ceil(0.995 * best)

    # device-resident outputs for the timed loop
    W = A.spin_words(N_SPINS)
    d_sp = torch.empty((CHAINS, W), dtype=torch.int64, device="cuda")
    d_sh = torch.empty(CHAINS, dtype=torch.int64, device="cuda")
    d_bs = torch.empty(CHAINS, dtype=torch.int64, device="cuda")
    d_fl = torch.empty(CHAINS, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")   # > L2 (126 MB)
    L = _lib.load()
    o = _lib.opts(engine)
    stream = torch.cuda.current_stream()
    trial_base = rank << 20

    def launch(step):
        _lib.check(L.anc_run_device(dev._h, tb._h, RUN_SEED, trial_base + step * CHAINS, CHAINS, o,
                                    d_sp.data_ptr(), d_sh.data_ptr(), d_bs.data_ptr(), d_fl.data_ptr(), None,
                                    stream.cuda_stream))

    for w in range(args.warmup):
        launch(1000 + w)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    succ_batches, succ, flips_total = 0, 0, 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev_index) as clk:
        for k in range(args.steps):
            flush.fill_(k)                         # L2 flush between timed iterations (not timed)
            ev[k][0].record(stream)
            launch(k)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    # success statistics of the timed batches (rerun readback: results of the last batch are on the device; recompute
    # all batches' cuts through the host API so that every timed batch is scored)
    for k in range(args.steps):
        r = A.run(dev, tb, RUN_SEED, trial_base + k * CHAINS, CHAINS, engine=engine)
        c = r.cuts(sumw)
        s = int((c >= target).sum())
        succ += s; succ_batches += int(s > 0); flips_total += int(r.flips.sum())
    t_batch_ms = sum(ms) / len(ms)
    if dist:
        t = torch.tensor([t_batch_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_batch_ms = float(t.item())

    # e2e: the same batch through the public C ABI with host outputs (tables uploaded from host each step,
    # results read back to host each step)
    fourT_np = tb.arrays()
    e2e_ms = []
    torch.cuda.synchronize()
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        tbk = A.Tables.from_arrays(**fourT_np)
        r = A.run(dev, tbk, RUN_SEED, trial_base + k * CHAINS, CHAINS, engine=engine)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            e2e_ms.append(1000.0 * dt)
    e2e_t = sum(e2e_ms) / len(e2e_ms)
    if dist:
        t = torch.tensor([e2e_t], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    h2d = SCHED["S"] * (4 + 4 + 8 + 4)
    d2h = CHAINS * (W * 8 + 8 * 3)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    S = SCHED["S"]
    anneals = CHAINS * ws
    value = anneals / (t_batch_ms / 1000.0)
    B = CHAINS
    nb = args.steps
    P_batch = succ_batches / nb
    p = succ / (B * nb)
    # roofline: algorithmic bytes of the bit-column update per launch (flipped rows x ceil(N/8) bytes, K = 1) plus
    # fields (8 B/spin/step) and spins (N/4 B/step), per anneal-step, summed over the batch
    mean_flips = flips_total / (B * nb)              # per anneal (whole schedule)
    alg_bytes = B * (mean_flips * math.ceil(N_SPINS / 8) + S * (8 * N_SPINS + N_SPINS / 4))
    hbm, _, peak_kind = measured_peaks()
    achieved = alg_bytes / (t_batch_ms / 1000.0) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "anneals/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_batch_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"N={N_SPINS} +-1 complete graph (seed {INSTANCE_SEED}), {CHAINS} concurrent anneals "
                               f"per GPU, S={S} counted Onsager lambda 1.05 ramp, t0 30 t1 5 q 4",
                   "engine": engine, "n": N_SPINS, "anneals_per_gpu": CHAINS, "S": S, "l2": "flushed between steps",
                   "parallelism": f"replicas x{ws}"},
        "tts99_us": {"primary": 1000.0 * tts99(P_batch, t_batch_ms), "secondary": 1000.0 * tts99_secondary(p, B, t_batch_ms),
                     "target_cut": target, "best_cut": best, "p": p, "P_batch": P_batch, "t_batch_us": 1000 * t_batch_ms},
        "us_per_anneal_step": 1000.0 * t_batch_ms / S, "ns_per_chain_step": 1e6 * t_batch_ms / (S * B),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": profile_traffic(f"plain_{engine}"), "peak_kind": peak_kind,
                     "note": "bit-column algorithmic bytes; J is L2-resident so the HBM copy peak is a lower bound "
                             "of the roof"},
        "e2e": {"value": anneals / (e2e_t / 1000.0), "unit": "anneals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_t},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="auto", choices=["auto", "plain", "tensor"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return bench_reference(args, ws, rank)
    return bench_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
