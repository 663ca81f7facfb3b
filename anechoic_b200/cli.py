"""Command-line drop-in for the reference's GPU runners sca_gpu / sca_gpu_bias (gpu/onsager_v2_20261007/src/
sca_gpu.cu:597-789, gpu/multibit_bias_20261008/src/sca_gpu_bias.cu:615-846): the same flags and the same output files,
so check_ref-style replays and the estimators (anechoic_b200.analyze) read them unchanged.

    python -m anechoic_b200.cli (--graph F | --gset F | --jint8 F) [--bias F] [--kbits K]
        --output PREFIX [--chains B] [--batches NB] [--seed S] [--offset O] [--trace 0|1]
        [--steps S --t0 T0 --t1 T1 --q Q --lambda L --tec-jv JV --tecT KAPPA --ramp]
        [--target CUT | --target-energy E] [--wide auto|0|1] [--check-fields 0|1] [--engine auto|plain|tensor|cluster]
        [--tensor-kind auto|int8|fp4] [--warmup W] [--info]

The reference's kernel-geometry flags (--cs, --groups, --clusters, --burn, --r, --preg) are accepted and recorded;
the engines here pick their own geometry. --warmup W (default 1) runs W untimed launches first, on trial ids
0xF0000000 + 65536 i far outside any cohort, with results discarded, as the reference CLIs do
(sca_gpu.cu:712-713), so batch 0 is timed like the rest. Success: cut >= --target (b = 0; default 33000 for a --graph
instance without bias, the reference's K2000 target) or energy <= --target-energy.

Files (PREFIX = --output):
  PREFIX.trials.jsonl    per anneal: batch, chain, trial_id, [cut, device_cut,] sum_sh, sum_bs, energy,
                         device_energy, [field_mismatches,] flips, success
  PREFIX.spins.bin       per anneal: spin_words(n) uint64, bit i = [s_i = +1]
  PREFIX.trace.bin       per anneal: S int32 n_lin (with --trace 1)
  PREFIX.batches.jsonl   per batch: batch, chains, trial_offset, device_ms, host_ms, successes
  PREFIX.summary.json    run parameters, successes, p, P_batch, Wilson 95 % intervals, TTS99, cut mismatches
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

from . import _lib, analyze
from .engine import DeviceInstance, Schedule, Tables, parse_schedule_flag, run, tdiv
from .instances import load, read_bias

GEOMETRY_FLAGS = ("--cs", "--groups", "--clusters", "--burn", "--r", "--preg")


def parse(argv):
    o = dict(jkind=None, jpath=None, bias=None, kbits=0, output=None, chains=1024, batches=1, seed=20261004, offset=0,
             trace=0, target=None, target_energy=None, wide="auto", check_fields=0, engine="auto", tensor_kind="auto",
             info=False,
             warmup=1, geometry={})
    sc = Schedule()
    a = 0
    while a < len(argv):
        k = argv[a]
        used = parse_schedule_flag(sc, argv, a)
        if used:
            a += used
            continue
        if k == "--info":
            o["info"] = True
            a += 1
            continue
        if a + 1 >= len(argv):
            raise ValueError("missing value for " + k)
        v = argv[a + 1]
        if k in ("--graph", "--gset", "--jint8"):
            o["jkind"], o["jpath"] = k[2:], v
        elif k == "--bias":
            o["bias"] = v
        elif k == "--kbits":
            o["kbits"] = int(v)
        elif k == "--output":
            o["output"] = v
        elif k in ("--chains", "--batches", "--trace", "--check-fields", "--warmup"):
            o[k[2:].replace("-", "_")] = int(v)
        elif k == "--seed":
            o["seed"] = int(v)
        elif k == "--offset":
            o["offset"] = int(v)
        elif k == "--target":
            o["target"] = int(v)
        elif k == "--target-energy":
            o["target_energy"] = int(v)
        elif k == "--wide":
            o["wide"] = v
        elif k == "--engine":
            o["engine"] = v
        elif k == "--tensor-kind":
            o["tensor_kind"] = v
        elif k in GEOMETRY_FLAGS:
            o["geometry"][k[2:]] = v
        else:
            raise ValueError("unknown argument " + k)
        a += 2
    return o, sc


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        o, sc = parse(argv)
        if not o["jkind"]:
            raise ValueError("one of --graph, --gset, --jint8 is required")
        inst = load(o["jkind"], o["jpath"])
        if o["bias"]:
            inst.bias = read_bias(o["bias"], inst.n)
        st = inst.stats()
        has_bias = inst.bias is not None and np.any(inst.bias != 0)
        target, target_e = o["target"], o["target_energy"]
        if target is None and target_e is None:
            if o["jkind"] == "graph" and not has_bias:
                target = 33000
            else:
                raise ValueError("--target CUT or --target-energy E required for this instance")
        if target is not None and has_bias:
            raise ValueError("--target (cut) is defined for b = 0 only; use --target-energy")
        dev = DeviceInstance(inst, kbits=o["kbits"]) if o["kbits"] else DeviceInstance(inst)
        tb = Tables.from_schedule(sc)
        wide = {"auto": "auto", "0": 0, "1": 1}[str(o["wide"])]
        if o["info"]:
            print(json.dumps(dict(n=inst.n, np=dev.info["np"], kbits=dev.info["kbits"], sparse=dev.info["sparse"],
                                  sumw=st["sumw"], steps=sc.S, range_plan=dev.range_plan(tb),
                                  version=_lib.load().anc_version().decode())))
            return 0
        if not o["output"]:
            raise ValueError("--output PREFIX required")
        out = o["output"]
        B, nb = o["chains"], o["batches"]
        dense = inst.to_dense().astype(np.float64) if not inst.is_sparse else None
        bias = inst.bias.astype(np.int64) if inst.bias is not None else np.zeros(inst.n, np.int64)
        succ = batch_succ = mism = fmis_total = 0
        dms, hms = [], []
        kernel = None
        gpu_before = gpu_status()
        for i in range(max(0, o["warmup"])):
            run(dev, tb, o["seed"], 0xF0000000 + 65536 * i, B, engine=o["engine"], wide=wide,
                tensor_kind=o["tensor_kind"])
        with open(out + ".trials.jsonl", "w") as ftr, open(out + ".batches.jsonl", "w") as fb, \
                open(out + ".spins.bin", "wb") as fsp, (open(out + ".trace.bin", "wb") if o["trace"] else _Null()) as ftc:
            for b in range(nb):
                off = o["offset"] + b * B
                h0 = time.perf_counter()
                r = run(dev, tb, o["seed"], off, B, trace=bool(o["trace"]), fields=bool(o["check_fields"]),
                        engine=o["engine"], wide=wide, tensor_kind=o["tensor_kind"])
                h1 = time.perf_counter()
                kernel = r.kernel
                dms.append(r.device_ms)
                hms.append(1000.0 * (h1 - h0))
                # independent host rescoring of every returned spin vector
                s = np.stack([inst.spins_pm(r.spins[c]) for c in range(B)]).astype(np.int64)
                sJs = _quadratic(inst, dense, s)
                cut_host = tdiv(st["sumw"] + sJs // 2, 2)
                e_host = -(sJs // 2) - (s * bias).sum(axis=1)
                cut_dev = r.cuts(st["sumw"])
                e_dev = r.energies()
                bs = 0
                for c in range(B):
                    ok = bool(cut_host[c] >= target) if target is not None else bool(e_host[c] <= target_e)
                    if not has_bias and cut_dev[c] != cut_host[c]:
                        mism += 1
                    if has_bias and e_dev[c] != e_host[c]:
                        mism += 1
                    rec = dict(batch=b, chain=c, trial_id=off + c)
                    if not has_bias:
                        rec.update(cut=int(cut_host[c]), device_cut=int(cut_dev[c]))
                    rec.update(sum_sh=int(r.sum_sh[c]), sum_bs=int(r.sum_bs[c]), energy=int(e_host[c]),
                               device_energy=int(e_dev[c]))
                    if o["check_fields"]:
                        fm = int(np.count_nonzero(r.fields[c] != inst.fields(r.spins[c])))
                        fmis_total += fm
                        rec["field_mismatches"] = fm
                    rec.update(flips=int(r.flips[c]), success=ok)
                    ftr.write(json.dumps(rec, separators=(",", ":")) + "\n")
                    succ += ok
                    bs += ok
                fsp.write(np.ascontiguousarray(r.spins, np.uint64).tobytes())
                if o["trace"]:
                    ftc.write(np.ascontiguousarray(r.trace, np.int32).tobytes())
                batch_succ += bs > 0
                fb.write(json.dumps(dict(batch=b, chains=B, trial_offset=off, device_ms=r.device_ms,
                                         host_ms=hms[-1], successes=bs), separators=(",", ":")) + "\n")
        summary = make_summary(o, sc, inst.n, kernel, succ, batch_succ, dms, hms, mism,
                               fmis_total if o["check_fields"] else None, target, target_e, gpu_before)
        with open(out + ".summary.json", "w") as f:
            f.write(json.dumps(summary) + "\n")
        print(json.dumps(summary))
        return 2 if mism or fmis_total else 0
    except (ValueError, OSError, _lib.AncError) as e:
        print("FAIL: " + str(e), file=sys.stderr)
        return 1


def make_summary(o: dict, sc: Schedule, n: int, kernel, succ: int, batch_succ: int, dms, hms, mism: int,
                 field_mismatches, target, target_e, gpu_before: str) -> dict:
    """The PREFIX.summary.json record. It carries every field the reference's runner writes
    (gpu/onsager_v2_20261007/src/sca_gpu.cu:769-781), so the reference's estimators (its analyze.py estimate(),
    which reads cs, groups, chains, batches, successes, device_ms_min / _max, gpu_before / _after among others)
    read this CLI's files unchanged. The reference's kernel-geometry flags (--cs, --groups, --clusters) are recorded
    as given (null when absent): the engines here pick their own geometry."""
    B, nb = o["chains"], o["batches"]
    t = sum(dms) / nb
    p, Pb = succ / (B * nb), batch_succ / nb
    geo = o["geometry"]

    def geo_int(k):
        try:
            return int(geo[k]) if k in geo else None
        except ValueError:
            return None

    return dict(device=_device_name(), uuid=_device_uuid(), n=n, engine=o["engine"], kernel=kernel,
                tensor_kind=o.get("tensor_kind", "auto"), geometry=geo, cs=geo_int("cs"), groups=geo_int("groups"),
                clusters=geo_int("clusters"), warmup=o["warmup"],
                chains=B, batches=nb, seed=o["seed"], trial_offset=o["offset"], steps=sc.S, t0=sc.t0, t1=sc.t1,
                q=sc.q, **{"lambda": sc.lam}, ramp=sc.ramp, tec_jv=sc.jv, tecT_kappa=sc.kappa, trace=o["trace"],
                target=target, target_energy=target_e, successes=succ, trials=B * nb, p=p,
                batches_with_success=batch_succ, P_batch=Pb, p_wilson95=list(analyze.wilson(succ, B * nb)),
                P_batch_wilson95=list(analyze.wilson(batch_succ, nb)), device_ms_mean=t,
                device_ms_min=min(dms), device_ms_max=max(dms), host_ms_mean=sum(hms) / nb,
                tts99_primary_ms=_finite(analyze.tts99(Pb, t)),
                tts99_secondary_ms=_finite(analyze.tts99_secondary(p, B, t)), cut_mismatches=mism,
                field_mismatches=field_mismatches, gpu_before=gpu_before, gpu_after=gpu_status())


def gpu_status() -> str:
    """One line of GPU state (utilisation, memory used, power, SM clock) from nvidia-smi, recorded before and after
    the batches as the reference's runner does (sca_gpu.cu:540-547); "?" where nvidia-smi is unavailable."""
    import subprocess
    try:
        r = subprocess.run(["nvidia-smi", "--id=0", "--query-gpu=utilization.gpu,memory.used,power.draw,clocks.sm",
                            "--format=csv,noheader"], capture_output=True, text=True, timeout=10)
        return r.stdout.strip() if r.returncode == 0 and r.stdout.strip() else "?"
    except (OSError, subprocess.SubprocessError):
        return "?"


def _quadratic(inst, dense, s: np.ndarray) -> np.ndarray:
    """s^T J s per row of s (int64), from the couplings on the host (dense matrix product in f64, exact for these
    integers, or the CSR rows)."""
    if dense is not None:
        return np.rint(((s.astype(np.float64) @ dense) * s).sum(axis=1)).astype(np.int64)
    rp, col, val = inst.to_csr()
    rows = np.repeat(np.arange(inst.n), np.diff(rp))
    v = val.astype(np.int64)
    return np.array([int((v * s[c, rows] * s[c, col]).sum()) for c in range(s.shape[0])], np.int64)


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def write(self, *_):
        pass


def _finite(x: float):
    return None if x == float("inf") else x


def _device_uuid() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return str(torch.cuda.get_device_properties(0).uuid)
    except Exception:       # informational only
        pass
    return ""


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0) if torch.cuda.is_available() else ""
    except Exception:       # device name is informational only
        return ""


if __name__ == "__main__":
    sys.exit(main())
