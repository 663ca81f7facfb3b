"""Host-side mirror of the reference's interface for the SCA anneal path, backed by the B200 engines.

Reference counterparts (paths relative to the reference project root):

* ``Schedule`` / ``build_tables`` / ``parse_schedule_flag`` -- v80host::Schedule, build_tables, parse_schedule_flag
  (gpu/onsager_v2_20261007/src/tables.hpp:18-55); ``Schedule.scale`` is mb::Sched::scale (mb_common.hpp:132-154).
* ``make_tables`` -- sca::make_tables (sca_ref.hpp:57-68).
* ``run_trial`` / ``run_trial_bias`` -- sca::run_trial / sca::run_trial_bias (sca_ref.hpp:101-155,
  sca_ref_bias.hpp:25-75): the same arguments and results, computed on the GPU.
* ``run`` -- one launch of sca_gpu / sca_gpu_bias over ``nchains`` trial ids (sca_gpu.cu:699-713).
* ``run_batch`` -- many (instance, schedule) jobs in one persistent launch.
* ``range_plan`` -- host::plan_ranges (gpu/multibit_bias_20261008/src/sca_gpu_bias.cu:543-557).

Errors raise ``AncError`` (the reference prints ``FAIL: ...`` and exits 1). Nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import AncError, check, load
from .instances import Instance, pad_spins, spin_words


@dataclasses.dataclass
class Schedule:
    """Annealing schedule (defaults of v80host::Schedule, tables.hpp:18-22). lam: counted Onsager gain; kappa:
    temperature-scaled correction (TEC-T); jv: TEC constant; scale: correction scale folded into lam / kappa."""

    S: int = 560
    t0: float = 30.0
    t1: float = 5.0
    q: float = 4.0
    lam: float = 0.0
    jv: float = 0.0
    kappa: float = 0.0
    ramp: bool = False
    scale: float = 1.0

    @property
    def mode(self) -> str:
        if self.kappa > 0:
            return "tecT"
        if self.lam != 0:
            return "onsager"
        if self.jv != 0:
            return "tec"
        return "plain"


def parse_schedule_flag(sc: Schedule, argv: Sequence[str], a: int) -> int:
    """Consume one schedule flag at argv[a] (tables.hpp:43-55). Returns the number of argv entries consumed (0 if
    argv[a] is not a schedule flag)."""
    k = argv[a]
    if k == "--ramp":
        sc.ramp = True
        return 1
    keys = {"--steps": ("S", int), "--t0": ("t0", float), "--t1": ("t1", float), "--q": ("q", float),
            "--lambda": ("lam", float), "--tec-jv": ("jv", float), "--tecT": ("kappa", float)}
    if k not in keys:
        return 0
    if a + 1 >= len(argv):
        raise ValueError("missing value for " + k)
    name, typ = keys[k]
    setattr(sc, name, typ(argv[a + 1]))
    return 2


class Tables:
    """Fixed-point per-step tables held on the device: fourT (Q16.16 of 4T), q (Q16.16), kcorr (Q8.24), kconst."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_arrays(cls, fourT, q, kcorr, kconst) -> "Tables":
        f = np.ascontiguousarray(fourT, np.int32); qq = np.ascontiguousarray(q, np.int32)
        kc = np.ascontiguousarray(kcorr, np.int64); ks = np.ascontiguousarray(kconst, np.int32)
        S = len(f)
        if not (len(qq) == len(kc) == len(ks) == S):
            raise ValueError("table arrays must have equal length")
        L = load()
        h = C.c_void_p()
        check(L.anc_tables_create(f.ctypes.data, qq.ctypes.data, kc.ctypes.data, ks.ctypes.data, S, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_schedule(cls, sc: Schedule) -> "Tables":
        L = load()
        h = C.c_void_p()
        check(L.anc_tables_from_schedule(sc.S, sc.t0, sc.t1, sc.q, sc.lam, sc.jv, sc.kappa, int(sc.ramp), sc.scale,
                                         C.byref(h)))
        return cls(h.value)

    @property
    def S(self) -> int:
        return load().anc_tables_steps(self._h)

    def arrays(self) -> dict:
        S = self.S
        f = np.zeros(S, np.int32); q = np.zeros(S, np.int32); kc = np.zeros(S, np.int64); ks = np.zeros(S, np.int32)
        check(load().anc_tables_read(self._h, f.ctypes.data, q.ctypes.data, kc.ctypes.data, ks.ctypes.data))
        return dict(fourT=f, q=q, kcorr=kc, kconst=ks)

    @property
    def onsager(self) -> bool:
        """True when the correction depends on n_lin (counted mode)."""
        return bool(np.any(self.arrays()["kcorr"] != 0))

    def __del__(self):
        lib = getattr(_lib, "_lib", None) if _lib is not None else None
        if getattr(self, "_h", None) and lib is not None and self._h.value:
            lib.anc_tables_destroy(self._h)
            self._h = C.c_void_p()


def build_tables(sc: Schedule) -> Tables:
    """v80host::build_tables (scale == 1) / mb::tables, bit-identical fixed-point tables on the device."""
    return Tables.from_schedule(sc)


def make_tables(T, q, lam, tec_jv: float = 0.0) -> Tables:
    """sca::make_tables (sca_ref.hpp:57-68) from explicit per-step T, q, lambda."""
    T = np.asarray(T, np.float64); q = np.asarray(q, np.float64); lam = np.asarray(lam, np.float64)
    S = len(T)
    fourT = np.array([int(_llround(4.0 * T[t] * 65536.0)) for t in range(S)], np.int32)
    qq = np.array([int(_llround(q[t] * 65536.0)) for t in range(S)], np.int32)
    kcorr = np.array([0 if t == 0 else int(_llround(lam[t] / (2.0 * T[t - 1]) * 16777216.0)) for t in range(S)], np.int64)
    kconst = np.array([0 if t == 0 else int(_llround(-tec_jv * 65536.0)) for t in range(S)], np.int32)
    return Tables.from_arrays(fourT, qq, kcorr, kconst)


def _llround(x: float) -> int:
    """C llround: round half away from zero."""
    import math
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


class DeviceInstance:
    """Couplings (and bias) resident on the GPU. Dense instances are packed into 1/2/4-bit planes (kbits=0 picks the
    smallest fitting: 1 for a +-1 complete graph); sparse ones keep CSR rows."""

    def __init__(self, inst: Instance, kbits: int = 0, sparse: Optional[bool] = None):
        self.inst = inst
        L = load()
        h = C.c_void_p()
        b = inst.bias
        bptr = b.ctypes.data if b is not None else None
        use_sparse = inst.is_sparse if sparse is None else sparse
        if use_sparse:
            rp, col, val = inst.to_csr()
            self._keep = (rp, col, val)
            check(L.anc_instance_create_csr(inst.n, rp.ctypes.data, col.ctypes.data, val.ctypes.data, bptr, C.byref(h)))
        else:
            d = inst.to_dense()
            check(L.anc_instance_create(d.ctypes.data, inst.n, kbits, bptr, C.byref(h)))
        self._h = h
        info = _lib.InstanceInfo()
        check(L.anc_instance_get_info(self._h, C.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in _lib.InstanceInfo._fields_}

    @property
    def n(self) -> int:
        return self.info["n"]

    def range_plan(self, tb: Tables) -> dict:
        ok = C.c_int(); hc = C.c_int32()
        check(load().anc_range_plan(self._h, tb._h, C.byref(ok), C.byref(hc)))
        return dict(plain_ok=bool(ok.value), hclamp=hc.value)

    def __del__(self):
        lib = getattr(_lib, "_lib", None) if _lib is not None else None
        if getattr(self, "_h", None) and lib is not None and self._h.value:
            lib.anc_instance_destroy(self._h)
            self._h = C.c_void_p()


@dataclasses.dataclass
class RunResult:
    """Per-chain results of one launch (trial ids trial_offset + c). spins: [nchains, spin_words(n)] uint64."""

    n: int
    trial_offset: int
    spins: np.ndarray
    sum_sh: np.ndarray
    sum_bs: np.ndarray
    flips: np.ndarray
    trace: Optional[np.ndarray] = None
    fields: Optional[np.ndarray] = None
    device_ms: float = 0.0
    profile: Optional[dict] = None
    kernel: Optional[str] = None     # "plain", "plain-cluster", "tensor-int8" or "tensor-fp4"

    def cuts(self, sumw: int) -> np.ndarray:
        """Device cut = (sumw + sum_sh / 2) / 2 with C++ truncating division (sca_ref.hpp:153)."""
        return tdiv(sumw + tdiv(self.sum_sh.astype(np.int64), 2), 2)

    def energies(self) -> np.ndarray:
        """E = -(sum_sh + sum_bs) / 2 (C++ truncation; sca_gpu_bias.cu:752)."""
        return tdiv(-(self.sum_sh.astype(np.int64) + self.sum_bs.astype(np.int64)), 2)


def tdiv(a, b: int):
    """Integer division truncating toward zero (C++ semantics)."""
    a = np.asarray(a, np.int64)
    return np.where(a >= 0, a // b, -((-a) // b))


def run(dev: DeviceInstance, tb: Tables, seed: int, trial_offset: int, nchains: int, trace: bool = False,
        fields: bool = False, engine: str = "auto", wide="auto", profile: bool = False,
        tensor_kind: str = "auto", flip_fraction: Optional[float] = None) -> RunResult:
    """nchains anneals (trial ids trial_offset .. trial_offset + nchains - 1) in one launch. engine: "auto",
    "plain" (one CTA per anneal), "cluster" (one anneal per 8-CTA cluster; dense 1-bit couplings, n <= 2048) or
    "tensor" (replicas sharing J). "auto" runs the engine with the least estimated device time (auto_estimate);
    flip_fraction (flips per spin per step) overrides the fraction it assumes, which is otherwise what the last run
    of these tables on this instance saw. profile=True records the tensor engine's per-phase cycle counters
    (RunResult.profile); tensor_kind picks the tensor engine's operand format ("auto", "int8", "fp4")."""
    L = load()
    n = dev.n
    W = spin_words(n)
    spins = np.zeros((nchains, W), np.uint64)
    sh = np.zeros(nchains, np.int64); bs = np.zeros(nchains, np.int64); fl = np.zeros(nchains, np.int64)
    S = tb.S
    tr = np.zeros((nchains, S), np.int32) if trace else None
    hf = np.zeros((nchains, n), np.int32) if fields else None
    o = _lib.opts(engine, wide, profile, tensor_kind, flip_fraction)
    args = (dev._h, tb._h, C.c_uint64(seed), C.c_uint32(trial_offset), nchains, C.byref(o), spins.ctypes.data,
            sh.ctypes.data, bs.ctypes.data, fl.ctypes.data, tr.ctypes.data if trace else None)
    if fields:
        check(L.anc_run_fields(*args, hf.ctypes.data))
    else:
        check(L.anc_run(*args))
    res = RunResult(n=n, trial_offset=trial_offset, spins=spins, sum_sh=sh, sum_bs=bs, flips=fl, trace=tr, fields=hf,
                    device_ms=L.anc_last_device_ms(), kernel=_lib.last_kernel())
    if profile:
        res.profile = _lib.last_profile()
    return res


_ENGINE_NAMES = {v: k for k, v in _lib.ENGINES.items()}


def auto_estimate(n: int, kbits: int, nchains: int, S: int, flip_fraction: float, per_wave: dict,
                  fp4: bool = False) -> dict:
    """The cost model behind engine="auto", host-only: estimated device time (ms) of one launch on each engine
    available (per_wave: anneals each engine advances at once, e.g. {"plain": 148, "tensor": 1152, "cluster": 15}),
    and under "pick" the engine with the least."""
    w = (C.c_int * 4)(0, *(int(per_wave.get(e, 0)) for e in ("plain", "tensor", "cluster")))
    us = (C.c_double * 4)()
    e = load().anc_auto_estimate(n, kbits, nchains, S, float(flip_fraction), int(bool(fp4)), w, us)
    if e < 0:
        check(e)
    out = {_ENGINE_NAMES[i]: us[i] / 1000.0 for i in (1, 2, 3) if us[i] >= 0}
    out["pick"] = _ENGINE_NAMES[e]
    return out


def auto_choice(dev: DeviceInstance, tb: Tables, nchains: int, flip_fraction: Optional[float] = None) -> dict:
    """The engine engine="auto" would run for run(dev, tb, ..., nchains), with the estimates (ms), the anneals per
    wave of each engine on this device and the flip fraction it assumed."""
    us = (C.c_double * 4)()
    w = (C.c_int * 4)()
    phi = C.c_double()
    o = _lib.opts("auto", flip_fraction=flip_fraction)
    e = load().anc_auto_choice(dev._h, tb._h, nchains, C.byref(o), us, w, C.byref(phi))
    if e < 0:
        check(e)
    names = ("plain", "tensor", "cluster")
    return {"pick": _ENGINE_NAMES[e], "ms": {k: us[i + 1] / 1000.0 for i, k in enumerate(names) if us[i + 1] >= 0},
            "per_wave": {k: w[i + 1] for i, k in enumerate(names)}, "flip_fraction": phi.value}


def run_batch(jobs: List[dict], engine: str = "auto", wide="auto") -> List[RunResult]:
    """Many jobs in one persistent launch; each job is dict(dev=DeviceInstance, tb=Tables, seed, trial_offset, nchains,
    trace=False). Returns one RunResult per job."""
    L = load()
    arr = (_lib.Job * len(jobs))()
    outs = []
    for k, j in enumerate(jobs):
        dev, tb, nc = j["dev"], j["tb"], int(j["nchains"])
        W = spin_words(dev.n)
        r = RunResult(n=dev.n, trial_offset=int(j.get("trial_offset", 0)), spins=np.zeros((nc, W), np.uint64),
                      sum_sh=np.zeros(nc, np.int64), sum_bs=np.zeros(nc, np.int64), flips=np.zeros(nc, np.int64),
                      trace=np.zeros((nc, tb.S), np.int32) if j.get("trace") else None)
        outs.append(r)
        a = arr[k]
        a.inst, a.tb = dev._h.value, tb._h.value
        a.seed, a.trial_offset, a.nchains = int(j["seed"]), r.trial_offset, nc
        a.spins, a.sum_sh, a.sum_bs, a.flips = (r.spins.ctypes.data, r.sum_sh.ctypes.data, r.sum_bs.ctypes.data,
                                                r.flips.ctypes.data)
        a.trace = r.trace.ctypes.data if r.trace is not None else None
    o = _lib.opts(engine, wide)
    check(L.anc_run_batch(len(jobs), arr, C.byref(o)))
    ms = L.anc_last_device_ms()
    for r in outs:
        r.device_ms = ms
    return outs


# ---- golden-model-shaped entry points (same arguments and results as sca::run_trial / run_trial_bias) ----
@dataclasses.dataclass
class Result:
    spins: np.ndarray     # spin_words(n) uint64
    cut: int
    flips: int
    n_lin: Optional[np.ndarray]


@dataclasses.dataclass
class ResultBias:
    spins: np.ndarray
    sum_sh: int
    sum_bs: int
    flips: int
    n_lin: Optional[np.ndarray]


def run_trial_bias(n: int, dense: np.ndarray, bias: Optional[np.ndarray], tb: Tables, seed: int, trial: int,
                   trace: bool = False, engine: str = "auto") -> ResultBias:
    """sca::run_trial_bias on the GPU (dense: n x n int8; bias: n int32 or None)."""
    dev = DeviceInstance(Instance(n=n, dense=np.asarray(dense, np.int8)[:n, :n], bias=bias))
    r = run(dev, tb, seed, trial, 1, trace=trace, engine=engine)
    return ResultBias(spins=r.spins[0], sum_sh=int(r.sum_sh[0]), sum_bs=int(r.sum_bs[0]), flips=int(r.flips[0]),
                      n_lin=r.trace[0] if trace else None)


def run_trial(inst: Instance, tb: Tables, seed: int, trial: int, trace: bool = False, engine: str = "auto") -> Result:
    """sca::run_trial on the GPU: cut = (sumw + sum_sh / 2) / 2."""
    dev = DeviceInstance(inst)
    r = run(dev, tb, seed, trial, 1, trace=trace, engine=engine)
    return Result(spins=r.spins[0], cut=int(r.cuts(dev.info["sumw"])[0]), flips=int(r.flips[0]),
                  n_lin=r.trace[0] if trace else None)
