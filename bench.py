#!/usr/bin/env python3
"""Benchmark of the SCA anneal path on B200: anneals/s and TTS99 to the target cut, one JSON line (rank 0).

Workload (one "step" = one batch): the N = 2000 +-1 complete graph (J_xy = J_yx iid uniform +-1, generator seed
20261004), 1024 concurrent anneals per GPU (trial ids rank*2^20 + step*1024 + c), counted Onsager correction
lambda = 1.05 with ramp, reference default schedule t0 = 30, t1 = 5, q = 4, S = 1000 steps, seed 20261004.
Target cut: 0.995 x the best cut of 1000 long anneals (S = 5000, same correction) of the same instance, run on the
exact engine outside the timed region. TTS99: primary t_batch ln(0.01)/ln(1 - P_batch), secondary
t_batch ln(0.01)/(B ln(1 - p)) (reference estimators, gpu/onsager_v2_20261007/src/analyze.py:15-47). Outside the
timed region the same schedule also runs at step budgets S = 100 ... 2000 ("tts99_by_budget": device time per batch,
success probability and secondary TTS99 per budget).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--engine auto|plain|tensor|cluster] [--tensor-kind auto|int8|fp4]
                  [--impl ours|reference]

--impl reference times the reference's own CPU golden model (sca::run_trial_bias compiled unmodified into
oracle/_ref/libscaref.so) on all host threads over a bounded sample of the same workload.

Besides the headline (one rank, N = 1), the line carries:
  cpu_baseline   the golden model on the host cores over the first anneals of the LAST TIMED BATCH (same trial ids),
                 and the numba float models of the engine (oracle/float_models.py) on the same host;
  parity         that sample compared bit for bit with the timed launch's own outputs (spins, sum s*h, flips);
  plain_engine   the bit-column engine on the same batches, with its roofline;
  single_anneal  config 1: one anneal, device time per step, single-chain TTS99, checked against the restatement;
  configs        config 3 (sparse51), config 5 (dense16k) and config 4 (meanfield), each with its roofline.
"""
from __future__ import annotations

import argparse
import ctypes as C
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
BUDGETS = (100, 200, 500, 1000, 2000)   # the metric's step budgets (S) for the TTS99 sweep
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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
    """(HBM copy GB/s, bf16 GEMM TFLOP/s burst, bf16 sustained, "measured" | "fallback")."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        bf = d.get("bf16_tflops", 1590.0)
        return d.get("hbm_gbs", 6650.0), bf, d.get("bf16_tflops_sustained", bf), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def profile_traffic(kernel: str):
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    e = d.get(kernel)
    return e.get("bytes_per_launch") if e else None


def stream_traffic(S: int):
    """DRAM bytes per launch of the streaming kernel at S steps: the committed capture (S = 20) scaled by the field
    updates, since J is read once per update (profiles/traffic.json)."""
    b = profile_traffic("tensor_stream_kernel")
    return None if b is None else b * (S + 1) / 21.0


def finite(obj):
    """The JSON line holds no inf or nan (strict JSON): a non-finite number (e.g. TTS99 with no success) becomes null."""
    if isinstance(obj, float):
        return obj if math.isfinite(obj) else None
    if isinstance(obj, dict):
        return {k: finite(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [finite(v) for v in obj]
    return obj


def tts99(P: float, t: float) -> float:
    if P >= 1.0:
        return t
    if P <= 0.0:
        return math.inf
    return t * math.log(0.01) / math.log(1.0 - P)


def tts99_secondary(p: float, B: int, t: float) -> float:
    """Secondary TTS99 with B anneals per batch of time t. When every anneal succeeds (p = 1) it is one anneal's share
    of the batch, t / B (the reference's per-trial estimators return one trial's time there,
    research/reaim_benchmarks_20261008/analyze.py:83), not 0."""
    if p <= 0.0:
        return math.inf
    if p >= 1.0:
        return t / B
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
    print(json.dumps(finite(line)))
    return 0


def cpu_baseline_sample(trial_offset: int, expected=None, budget_s: float = 15.0):
    """The reference's CPU golden model on the host cores (rank 0, N = 1 only): anneals/s on a bounded sample, and the
    in-bench parity check. The sample is the first anneals of one timed GPU batch: trial ids trial_offset + c,
    c = 0, 1, ... in rounds of one anneal per host thread until about budget_s seconds have passed. expected =
    (spins [B, W] uint64, sum_sh [B], flips [B]) of that batch as the timed launch left them in device memory; every
    anneal of the sample is compared with them bit for bit."""
    import numpy as np
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
    checked = mism = 0
    first_bad = None

    def compare(res, c0, k):
        nonlocal checked, mism, first_bad
        if expected is None:
            return
        sp, sh, fl = expected
        W = sp.shape[1]
        for c in range(k):
            ok = (np.array_equal(res["spins"][c][:W], sp[c0 + c]) and int(res["sum_sh"][c]) == int(sh[c0 + c])
                  and int(res["flips"][c]) == int(fl[c0 + c]))
            checked += 1
            if not ok:
                mism += 1
                first_bad = first_bad if first_bad is not None else c0 + c

    limit = CHAINS if expected is None else min(CHAINS, expected[0].shape[0])
    t0 = time.perf_counter()
    compare(run(cores, trial_offset), 0, cores)
    first = time.perf_counter() - t0
    reps = max(1, min(int(budget_s / max(first, 1e-3)), limit // cores - 1))
    t0 = time.perf_counter()
    for r in range(reps):
        compare(run(cores, trial_offset + (r + 1) * cores), (r + 1) * cores, cores)
    dt = time.perf_counter() - t0
    out = {"value": reps * cores / dt, "unit": "anneals/s", "cores": cores, "kind": kind,
           "sample": f"{reps * cores} anneals (N={N_SPINS}, S={SCHED['S']}, counted Onsager) on {cores} threads, "
                     f"{dt:.1f} s; trial ids of the last timed GPU batch"}
    parity = None
    if expected is not None:
        parity = {"checked": checked, "mismatches": mism, "checker": kind, "batch": "last timed batch",
                  "trial_ids": f"{trial_offset} .. {trial_offset + checked - 1}",
                  "compared": "spins, sum s*h, flips (bit-exact)"}
        if first_bad is not None:
            parity["first_mismatch_chain"] = first_bad
    return out, parity


def numba_baselines(budget_s: float = 6.0):
    """The reference's numba float models of the engine, restated (oracle/float_models.py), on the host cores:
    the fused integer model with one anneal per thread, and the sequential float32 model on one thread."""
    from anechoic_b200 import instances as I
    from oracle import float_models as F
    inst = I.complete_pm1(N_SPINS, INSTANCE_SEED)
    return F.time_models(inst.dense, SCHED["S"], SCHED["t0"], SCHED["t1"], SCHED["q"], SCHED["lam"], SCHED["ramp"],
                         os.cpu_count() or 1, budget_s=budget_s)


# ------------------------------------------------------------------------------------------------------ our arm
KERNEL_NAMES = {"plain": "plain_kernel", "tensor-int8": "tensor_res_kernel", "tensor-fp4": "tensor_fp4_kernel"}


def roofline(kernel: str, t_launch_ms: float, B: int, S: int, mean_flips: float, np_pad: int):
    """Roofline of the dominant kernel for one launch of B anneals x S steps.
    plain: algorithmic bytes = B x (flipped rows x ceil(N/8) B of 1-bit couplings + S x (8 N B of fields + N/4 B of
    spin bits)), against the measured HBM copy bandwidth (J is L2-resident, so HBM is a lower bound of the roof).
    tensor: dense contraction ops = 2 x NP^2 x B x (S + 1) (every column of dS, the initial field included), against
    the sm_100 dense rate of the operand format relative to the measured bf16 GEMM: int8 2x, fp4 (e2m1) 4x."""
    hbm, bf16, _, peak_kind = measured_peaks()
    if kernel == "plain":
        alg = B * (mean_flips * math.ceil(N_SPINS / 8) + S * (8 * N_SPINS + N_SPINS / 4))
        ach = alg / (t_launch_ms / 1000.0) / 1e9
        return {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": profile_traffic(KERNEL_NAMES[kernel]), "peak_kind": peak_kind,
                "algorithmic_per_launch": alg, "kernel": KERNEL_NAMES[kernel],
                "note": "bit-column algorithmic bytes; J is L2-resident so the HBM copy peak is a lower bound of the roof"}
    mult = 4.0 if kernel == "tensor-fp4" else 2.0
    ops = 2.0 * np_pad * np_pad * B * (S + 1)
    ach = ops / (t_launch_ms / 1000.0) / 1e12
    peak = mult * bf16
    return {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "traffic": profile_traffic(KERNEL_NAMES[kernel]), "peak_kind": f"{peak_kind} bf16 x {mult:g}",
            "algorithmic_per_launch": ops, "kernel": KERNEL_NAMES[kernel],
            "useful_fraction": mean_flips / (N_SPINS * S),
            "note": f"{'fp4' if mult == 4 else 'int8'} dense ops (tera-ops/s), 2 NP^2 per replica-step; peak = "
                    f"{mult:g} x measured bf16 GEMM (sm_100 dense rate ratio)"}


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
    engine, kind = args.engine, args.tensor_kind

    # target cut (outside the timed region): best of 1000 long anneals on the exact engine
    ttb = A.Tables.from_schedule(A.Schedule(**TARGET_SCHED))
    tr = A.run(dev, ttb, RUN_SEED, 0xE0000000, TARGET_ANNEALS, engine=engine, tensor_kind=kind)
    best = int(tr.cuts(sumw).max())
    target = math.ceil(0.995 * best)

    W = A.spin_words(N_SPINS)
    d_sp = torch.empty((CHAINS, W), dtype=torch.int64, device="cuda")
    d_sh = torch.empty(CHAINS, dtype=torch.int64, device="cuda")
    d_bs = torch.empty(CHAINS, dtype=torch.int64, device="cuda")
    d_fl = torch.empty(CHAINS, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")   # > L2 (126 MB)
    L = _lib.load()
    stream = torch.cuda.current_stream()
    from anechoic_b200 import replicas
    trial_base = replicas.trial_base(rank)

    def timed(eng, knd, steps, warmup, clocks=False, nchains=CHAINS, base=trial_base):
        """Device-timed launches (inputs resident, outputs on the device) of nchains anneals with trial ids
        base + step * nchains + c; returns per-launch ms, the kernel, the clock sampler and the last launch's
        outputs (spins, sum s*h, flips) copied to the host after the timed region."""
        o = _lib.opts(eng, tensor_kind=knd)

        def launch(step):
            _lib.check(L.anc_run_device(dev._h, tb._h, RUN_SEED, base + step * nchains, nchains, o,
                                        d_sp.data_ptr(), d_sh.data_ptr(), d_bs.data_ptr(), d_fl.data_ptr(), None,
                                        stream.cuda_stream))

        for w in range(warmup):
            launch(1000 + w)
        torch.cuda.synchronize()
        kern = _lib.last_kernel()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(dev_index) if clocks else None
        if clk:
            clk.__enter__()
        for k in range(steps):
            flush.fill_(k)                         # L2 flush between timed iterations (not timed)
            ev[k][0].record(stream)
            launch(k)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__(None, None, None)
        if dist:
            dist.barrier()
        last = (d_sp[:nchains].cpu().numpy().view(np.uint64).copy(), d_sh[:nchains].cpu().numpy().copy(),
                d_fl[:nchains].cpu().numpy().copy())
        return [a.elapsed_time(b) for a, b in ev], kern, clk, last

    def scored(eng, knd, steps):
        """Success statistics of the timed batches, recomputed through the host API (same trial ids)."""
        succ, succ_batches, flips_total = 0, 0, 0
        for k in range(steps):
            r = A.run(dev, tb, RUN_SEED, trial_base + k * CHAINS, CHAINS, engine=eng, tensor_kind=knd)
            c = r.cuts(sumw)
            s_ = int((c >= target).sum())
            succ += s_; succ_batches += int(s_ > 0); flips_total += int(r.flips.sum())
        return succ, succ_batches, flips_total

    max_over_ranks = replicas.reduce_max

    ms, kernel, clk, last = timed(engine, kind, args.steps, args.warmup, clocks=True)
    t_batch_ms = max_over_ranks(sum(ms) / len(ms))
    succ, succ_batches, flips_total = replicas.reduce_sum(scored(engine, kind, args.steps))
    np_pad = L.anc_np(N_SPINS)

    # the plain (bit-column) engine on the same batches, for the batched-vs-plain comparison of the metric
    plain = None
    if kernel != "plain" and not args.no_plain:
        pms, _, _, _ = timed("plain", "auto", args.steps, args.warmup)
        p_ms = max_over_ranks(sum(pms) / len(pms))
        p_succ, p_sb, p_flips = replicas.reduce_sum(scored("plain", "auto", args.steps))
        plain = {"anneals_per_s": CHAINS * ws / (p_ms / 1000.0), "ms_per_step": p_ms,
                 "tts99_us_primary": 1000.0 * tts99(p_sb / (args.steps * ws), p_ms),
                 "tts99_us_secondary": 1000.0 * tts99_secondary(p_succ / (CHAINS * args.steps * ws), CHAINS, p_ms),
                 "roofline": roofline("plain", p_ms, CHAINS, SCHED["S"], p_flips / (CHAINS * args.steps * ws),
                                      np_pad)}

    # the metric's step budgets: the same schedule stretched to S = 100 ... 2000, two batches each, device-timed (the
    # launch's CUDA events) and scored against the same target; secondary TTS99 per budget (outside the timed region)
    budgets = {}
    if not args.no_budget_sweep:
        for Sb in BUDGETS:
            tbb = A.Tables.from_schedule(A.Schedule(**dict(SCHED, S=Sb)))
            A.run(dev, tbb, RUN_SEED, 0xD0000000, CHAINS, engine=engine, tensor_kind=kind)
            bms, bs = [], 0
            for k in range(2):
                r = A.run(dev, tbb, RUN_SEED, 0xD0000000 + (k + 1) * CHAINS, CHAINS, engine=engine, tensor_kind=kind)
                bms.append(r.device_ms)
                bs += int((r.cuts(sumw) >= target).sum())
            pb, tb_ms = bs / (2 * CHAINS), sum(bms) / len(bms)
            tts = 1000.0 * tts99_secondary(pb, CHAINS, tb_ms)
            budgets[str(Sb)] = {"ms_per_batch": tb_ms, "p": pb, "kernel": r.kernel,
                                "tts99_us_secondary": tts if math.isfinite(tts) else None}   # None: no success

    # e2e: the same batch through the public C ABI with host buffers -- schedule tables uploaded from host memory
    # and results (spins, sum s*h, sum b*s, flips) read back to host memory inside every timed step; the instance
    # (J, packed once by anc_instance_create) stays resident on the device across steps
    arrays = tb.arrays()
    # host buffers in pinned memory, as a caller that streams batches would hold them: the tables' four arrays in,
    # spins and the three per-anneal sums out
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    arrays_p = {}
    for key, v in arrays.items():
        arrays_p[key] = pinned(v.shape, {np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}[v.dtype])
        arrays_p[key][:] = v
    h_sp = pinned((CHAINS, W), torch.int64).view(np.uint64)
    h_sh, h_bs, h_fl = (pinned((CHAINS,), torch.int64) for _ in range(3))
    e2e_opts = _lib.opts(engine, tensor_kind=kind)
    e2e_ms, e2e_kernels = [], set()
    torch.cuda.synchronize()
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        tbk = A.Tables.from_arrays(**arrays_p)
        _lib.check(L.anc_run(dev._h, tbk._h, RUN_SEED, trial_base + k * CHAINS, CHAINS, C.byref(e2e_opts),
                             h_sp.ctypes.data, h_sh.ctypes.data, h_bs.ctypes.data, h_fl.ctypes.data, None))
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            e2e_ms.append(1000.0 * dt)
            e2e_kernels.add(_lib.last_kernel())
    e2e_t = max_over_ranks(sum(e2e_ms) / len(e2e_ms))
    h2d = SCHED["S"] * (4 + 4 + 8 + 4)
    d2h = CHAINS * (W * 8 + 8 * 3)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    S = SCHED["S"]
    anneals = CHAINS * ws
    value = anneals / (t_batch_ms / 1000.0)
    B, nb = CHAINS, args.steps * ws          # success counts are summed over ranks: ws batches per timed step
    P_batch = succ_batches / nb
    p = succ / (B * nb)
    mean_flips = flips_total / (B * nb)
    line = {
        "metric": METRIC, "value": value, "unit": "anneals/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_batch_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32" if kernel == "plain" else ("fp4-e2m1/f32" if kernel == "tensor-fp4"
                                                                         else "int8/int32"),
        "data": "synthetic",
        "config": {"workload": f"N={N_SPINS} +-1 complete graph (seed {INSTANCE_SEED}), {CHAINS} concurrent anneals "
                               f"per GPU, S={S} counted Onsager lambda 1.05 ramp, t0 30 t1 5 q 4",
                   "engine": engine, "kernel": kernel, "n": N_SPINS, "anneals_per_gpu": CHAINS, "S": S,
                   "l2": "flushed between steps", "parallelism": f"replicas x{ws}"},
        "tts99_us": {"primary": 1000.0 * tts99(P_batch, t_batch_ms), "secondary": 1000.0 * tts99_secondary(p, B, t_batch_ms),
                     "target_cut": target, "best_cut": best, "p": p, "P_batch": P_batch, "t_batch_us": 1000 * t_batch_ms},
        "plain_engine": plain,
        "tts99_by_budget": budgets or None,
        "us_per_anneal_step": 1000.0 * t_batch_ms / S, "ns_per_chain_step": 1e6 * t_batch_ms / (S * B),
        "ms_per_step_spread": [min(ms), max(ms)],
        "roofline": roofline(kernel, t_batch_ms, B, S, mean_flips, np_pad),
        "e2e": {"value": anneals / (e2e_t / 1000.0), "unit": "anneals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_t, "kernels": sorted(k for k in e2e_kernels if k),
                "same_kernel_as_timed": e2e_kernels == {kernel},
                "scope": "tables uploaded and results read back every step, from and into pinned host buffers; the "
                         "instance stays resident"},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if ws == 1 and not args.no_cpu_baseline:
        cpu, parity = cpu_baseline_sample(trial_base + (args.steps - 1) * CHAINS, last)
        line["cpu_baseline"] = cpu
        line["parity"] = parity
        if not args.no_numba:
            line["cpu_baseline"]["numba"] = numba_baselines()
    if ws == 1 and not args.no_extra:
        line["single_anneal"] = single_anneal(A, dev, tb, timed, p, sumw, target)
        extra = {}
        for name in ("sparse51", "dense16k", "meanfield"):
            extra[name] = run_extra(name, args, target=target)
        line["configs"] = extra
    print(json.dumps(finite(line)))
    if dist:
        dist.destroy_process_group()
    return 0


def single_anneal(A, dev, tb, timed, p, sumw, target):
    """Config 1: one anneal of the headline schedule on the engine AUTO picks for a single anneal, device-timed
    (CUDA events, 3 warm-up and 10 timed launches), bit-checked against the golden model on the same trial ids, with
    the single-chain TTS99 t ln(0.01) / ln(1 - p) from the headline batches' per-anneal success probability p (the
    anneals are identically distributed whatever engine runs them)."""
    import numpy as np
    ms, kern, _, last = timed("auto", "auto", 10, 3, nchains=1, base=0xC0000000)
    t = sum(ms) / len(ms)
    out = {"kernel": kern, "ms_per_anneal": t, "us_per_step": 1000.0 * t / SCHED["S"], "launches": len(ms),
           "ms_spread": [min(ms), max(ms)], "p": p,
           "tts99_us_single_chain": 1000.0 * tts99(p, t)}
    try:
        from oracle.oracle import Restatement
        R = Restatement()
        ref = R.run_batch(N_SPINS, R.tables(**SCHED), RUN_SEED, 0xC0000000 + 9, 1, dense=dev.inst.dense, trace=False)
        out["parity"] = {"checked": 1, "mismatches": int(not (np.array_equal(ref["spins"][0], last[0][0]) and
                                                              int(ref["sum_sh"][0]) == int(last[1][0]) and
                                                              int(ref["flips"][0]) == int(last[2][0])))}
    except (OSError, ImportError) as e:         # the checker could not load: say so, keep the timing
        out["parity"] = {"unavailable": str(e)}
    return out


# ------------------------------------------------------------------------------------------------ other workloads
EXTRA_DESC = {
    "sparse51": "51 synthetic sparse instances N=800..20000 (G-set-shaped classes, weights +1 or iid +-1, K=2 range, "
                "integer bias in [-2, 2]), 64 anneals each, S=1000 temperature-scaled kappa 2 ramp, ONE persistent "
                "launch of the plain engine (CSR path)",
    "dense16k": "N=16384 complete graph, J iid uniform in [-7, 7] (K=4), bias uniform in [-7, 7], 256 anneals, S=5000 "
                "counted Onsager lambda 1.05 ramp (the range plan's exact clamp active), tensor engine (J streamed)",
    "meanfield": "mean-field relaxation of the N=2000 +-1 instance: 64 replicas x 200 steps, f32 magnetisations, BF16 "
                 "J, f32 accumulation, forward and adjoint (checkpoint every 16 steps)",
}


def run_extra(name: str, args, steps: int = 3, warmup: int = 1, target=None) -> dict:
    """One of the other benchmark workloads, timed on the device (the library's CUDA events around each launch, or
    events on the stream), outside the headline's timed region, with its own roofline. meanfield also tunes the
    schedule on the relaxation and judges the tuned and the default schedule on the exact engine (1024 anneals each,
    same trial ids): p at the default schedule's median cut and, when given, at the headline's target cut."""
    import numpy as np
    import torch
    import anechoic_b200 as A
    from anechoic_b200 import instances as I
    hbm, bf16, bf16_sus, peak_kind = measured_peaks()
    if name == "meanfield":
        from anechoic_b200 import meanfield as M
        inst = I.complete_pm1(N_SPINS, INSTANCE_SEED)
        mf = M.MeanField(inst)
        S, R = 200, M.REPLICAS
        sch = M.SoftSchedule(S=S)
        theta = torch.tensor([30.0, math.log(6.0), 4.0, 0.0, 1.05], dtype=torch.float64, device="cuda")
        beta, q, u, w = sch.vectors(theta)
        sched = torch.stack([beta, q, u, w]).to(torch.float32).contiguous()
        m0 = mf.pad(M.initial_magnetisations(inst.n, R, 1))
        mprev = torch.zeros_like(m0)
        mprev[:, : inst.n] = 1.0
        g = torch.ones_like(m0)
        fw, bw = [], []
        for k in range(warmup + steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            out, ck = mf.forward_raw(sched, m0, mprev)
            e[1].record()
            mf.backward_raw(sched, ck, g)
            e[2].record()
            torch.cuda.synchronize()
            if k >= warmup:
                fw.append(e[0].elapsed_time(e[1]))
                bw.append(e[1].elapsed_time(e[2]))
        tf, tb_ = sum(fw) / len(fw), sum(bw) / len(bw)
        fl_f = 2.0 * inst.n * inst.n * R * S           # algorithmic: J m per step
        ach = fl_f / (tf / 1000.0) / 1e12
        ach_b = 2 * fl_f / (tb_ / 1000.0) / 1e12
        theta0 = (30.0, math.log(6.0), 4.0, 0.0, 1.05)
        t_tune = time.perf_counter()
        tuned, hist = M.tune(inst, S=S, R=R, theta0=theta0, iters=40, lr=0.01)
        t_tune = time.perf_counter() - t_tune
        thetas = {"default": torch.tensor(theta0, dtype=torch.float64), "tuned": tuned.cpu()}
        judged = M.judge(inst, S, thetas, nchains=CHAINS, seed=RUN_SEED, trial_offset=0xA0000000)
        if target is not None:
            judged = M.judge(inst, S, thetas, nchains=CHAINS, seed=RUN_SEED, trial_offset=0xA0000000,
                             targets={"median_default": judged["targets"]["median_first"],
                                      "headline_target": int(target)})
        return {"workload": EXTRA_DESC[name], "forward_ms": tf, "adjoint_ms": tb_, "replicas": R, "S": S,
                "tuning": {"iters": len(hist), "wall_s": t_tune, "soft_cut_first": hist[0][1],
                           "soft_cut_last": hist[-1][1]},
                "exact_engine_judgement": judged,
                "roofline": {"bound": "tensor", "achieved": ach, "peak": bf16_sus, "unit": "TFLOP/s",
                             "frac": ach / bf16_sus, "peak_kind": f"{peak_kind} bf16 sustained",
                             "algorithmic_per_launch": fl_f, "kernel": "mf_gemm_kernel (+ mf_fwd_kernel)",
                             "adjoint_achieved": ach_b, "adjoint_frac": ach_b / bf16_sus,
                             "note": "2 n^2 R FLOPs per forward step; the adjoint counts 2x that (recompute + J p)"}}
    if name == "sparse51":
        insts = [b() for _, b in I.sparse_classes_manifest()]
        sched = dict(S=1000, t0=6.0, t1=0.5, q=1.5, kappa=2.0, ramp=True)
        per = 64
    else:
        insts = [I.random_kbit(16384, 4, 20261009, pzero=0.0, bmax=7)]
        sched = dict(S=5000, t0=float(2 * np.sqrt(16384) * 4), t1=2.0, q=4.0, lam=1.05, ramp=True)
        per = 256
    devs = [A.DeviceInstance(i) for i in insts]
    tb = A.Tables.from_schedule(A.Schedule(**sched))
    eng = args.engine if args.engine != "cluster" else "auto"

    def launch(step):
        if len(devs) > 1:
            return A.run_batch([dict(dev=d, tb=tb, seed=RUN_SEED, trial_offset=(step << 12) + 64 * k, nchains=per)
                                for k, d in enumerate(devs)], engine=eng)
        return [A.run(devs[0], tb, RUN_SEED, step << 12, per, engine=eng)]

    kernel = None
    for w in range(warmup):
        kernel = launch(1000 + w)[0].kernel
    if len(devs) > 1:
        kernel = "plain"          # anc_run_batch runs the plain engine's persistent launch
    ms, flips = [], 0
    for k in range(steps):
        outs = launch(k)
        ms.append(outs[0].device_ms)
        flips += sum(int(o.flips.sum()) for o in outs)
    t = sum(ms) / len(ms)
    anneals = per * len(devs)
    S = sched["S"]
    mean_flips = flips / steps
    out = {"workload": EXTRA_DESC[name], "anneals_per_s": anneals / (t / 1000.0), "ms_per_launch": t,
           "ms_spread": [min(ms), max(ms)], "anneals": anneals, "S": S, "kernel": kernel, "launches": steps,
           "mean_flips_per_anneal_step": mean_flips / (anneals * S)}
    if kernel and kernel.startswith("tensor"):
        # dense int8 ops 2 NP^2 per replica-step (S + 1 field updates) against 2x the measured bf16 GEMM; J (NP^2
        # bytes) is streamed from HBM once per step for every pair of replica groups (256 anneals)
        npad = devs[0].info["np"]
        ops = 2.0 * npad * npad * anneals * (S + 1)
        jbytes = float(npad) * npad * (S + 1) * ((anneals + 255) // 256)
        a_ops = ops / (t / 1000.0) / 1e12
        a_j = jbytes / (t / 1000.0) / 1e9
        out["roofline"] = {"bound": "tensor", "achieved": a_ops, "peak": 2 * bf16_sus, "unit": "TFLOP/s",
                           "frac": a_ops / (2 * bf16_sus), "peak_kind": f"{peak_kind} bf16 sustained x 2",
                           "algorithmic_per_launch": ops, "kernel": "tensor_stream_kernel",
                           "hbm_j_stream": {"achieved": a_j, "peak": hbm, "unit": "GB/s", "frac": a_j / hbm},
                           "traffic": stream_traffic(S),
                           "note": "int8 dense ops (tera-ops/s), every column of dS counted"}
    else:
        # algorithmic bytes: coupling rows of flipped spins (CSR entries of 4 B) + fields (8 B) and spin bits
        # (1/4 B) per slot and step
        row_bytes = sum(4.0 * (len(i.col) / i.n) for i in insts) / len(insts)
        alg = mean_flips * row_bytes + sum(i.n for i in insts) * per * S * 8.25
        ach = alg / (t / 1000.0) / 1e9
        out["roofline"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                           "traffic": profile_traffic("plain_kernel_csr"),
                           "peak_kind": peak_kind, "algorithmic_per_launch": alg, "kernel": "plain_kernel",
                           "note": "CSR rows of flipped spins + fields + spin bits; rows are L2-resident, so the HBM "
                                   "copy peak is a lower bound of the roof"}
    return out


def bench_workload(args, ws, rank, local):
    """Opt-in single-GPU line for one of the other workloads (the default line carries all of them under
    "configs")."""
    import torch
    torch.cuda.set_device(local)
    with ClockSampler(local) as clk:
        res = run_extra(args.workload, args, steps=args.steps, warmup=args.warmup)
    line = {"metric": "anneals/s", "workload": args.workload, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "data": "synthetic", **res, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(finite(line)))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="auto", choices=["auto", "plain", "tensor", "cluster"])
    ap.add_argument("--tensor-kind", default="auto", choices=["auto", "int8", "fp4"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-engine comparison run")
    ap.add_argument("--no-budget-sweep", action="store_true", help="skip the TTS99 sweep over step budgets")
    ap.add_argument("--no-numba", action="store_true", help="skip the numba float-model CPU baselines")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the single-anneal and other-workload objects of the headline line")
    ap.add_argument("--workload", default="pm1", choices=["pm1", "sparse51", "dense16k", "meanfield"],
                    help="pm1: the headline line (default); the others print their own opt-in line")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return bench_reference(args, ws, rank)
    if args.workload != "pm1":
        return bench_workload(args, ws, rank, local)
    return bench_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
