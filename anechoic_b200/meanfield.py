"""Differentiable mean-field relaxation of the corrected SCA dynamics, for tuning annealing schedules.

The soft surrogate (per replica, t = 0 .. S-1, m in [-1, 1]^n):

    P_t     = J m_t + b + q_t m_t - gamma_t m_{t-1}
    gamma_t = u_t * sum_i (1 - m_t,i^2) + w_t
    m_{t+1} = tanh(P_t / (2 T_t))

is the tanh form of the reference's effective process (research/dmft_sca_20261004/dmft_torch.py:38-57) and the soft
version of the golden model's step (sca_ref.hpp:118-131): the exact engine flips with probability
(1 - clamp(s g / 2T)) / 2 for g = h + q s - corr s_prev, and its counted correction corr = lambda_t n_lin / (2 T_{t-1})
becomes u_t times the expected number of slots in the linear band. The forward pass and its adjoint are hand-written
sm_100a kernels behind the C ABI (J in BF16 on tcgen05, f32 magnetisations, checkpoints every 16 steps); this module
wraps them in a torch.autograd.Function and maps the five schedule parameters (T0, cooling rate, q0, q slope,
correction gain) onto the per-step vectors. A tuned schedule is judged only by the exact integer engine
(``SoftSchedule.tables``), which it never alters.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, load
from .instances import Instance

REPLICAS = 64          # replica rows of the kernels (MMA N); fewer replicas leave rows unused
CHECKPOINT = 16


def _bind(L):
    if getattr(L, "_mf_bound", False):
        return L
    vp, i = C.c_void_p, C.c_int
    L.anc_mf_create.argtypes = [vp, i, vp, C.POINTER(vp)]
    L.anc_mf_npad.argtypes = [vp]
    L.anc_mf_forward.argtypes = [vp, i, vp, vp, vp, vp, vp, vp]
    L.anc_mf_backward.argtypes = [vp, i, vp, vp, vp, vp, vp]
    L.anc_mf_check.argtypes = [vp, vp]
    L.anc_mf_set_wait_ns.argtypes = [vp, C.c_uint64]
    L.anc_mf_destroy.argtypes = [vp]
    L.anc_mf_destroy.restype = None
    L._mf_bound = True
    return L


class MeanField:
    """Device context of one instance (J in BF16, bias in f32) for the relaxation kernels."""

    def __init__(self, inst: Instance):
        L = _bind(load())
        if not torch.cuda.is_available():
            raise RuntimeError("the mean-field kernels need a CUDA device (there is no CPU fallback)")
        d = np.ascontiguousarray(inst.to_dense(), dtype=np.int8)
        b = None if inst.bias is None else np.ascontiguousarray(inst.bias, dtype=np.int32)
        h = C.c_void_p()
        check(L.anc_mf_create(d.ctypes.data, inst.n, b.ctypes.data if b is not None else None, C.byref(h)))
        self._h, self.n = h, inst.n
        self.npad = L.anc_mf_npad(h)
        self.inst = inst

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def forward_raw(self, sched: torch.Tensor, m0: torch.Tensor, mprev: torch.Tensor):
        """sched [4, S] f32 (beta, q, u, w) and m0 / mprev [64, npad] f32 on the device -> (m_S, checkpoints)."""
        L = load()
        S = sched.shape[1]
        ck = torch.empty((math.ceil(S / CHECKPOINT), 2, REPLICAS, self.npad), dtype=torch.float32, device="cuda")
        out = torch.empty((REPLICAS, self.npad), dtype=torch.float32, device="cuda")
        check(L.anc_mf_forward(self._h, S, sched.data_ptr(), m0.data_ptr(), mprev.data_ptr(), ck.data_ptr(),
                               out.data_ptr(), self._stream()))
        check(L.anc_mf_check(self._h, self._stream()))
        return out, ck

    def backward_raw(self, sched: torch.Tensor, ck: torch.Tensor, g_m: torch.Tensor) -> torch.Tensor:
        """dL/dm_S [64, npad] -> per-replica partials [S, 4, 64] of dL/d(beta, q, u, w)."""
        L = load()
        S = sched.shape[1]
        gs = torch.empty((S, 4, REPLICAS), dtype=torch.float32, device="cuda")
        check(L.anc_mf_backward(self._h, S, sched.data_ptr(), ck.data_ptr(), g_m.data_ptr(), gs.data_ptr(),
                                self._stream()))
        check(L.anc_mf_check(self._h, self._stream()))
        return gs

    def set_wait_ns(self, ns: int):
        """Limit of each device wait (default 2 s) before the kernels give up and report ANC_ETIMEOUT."""
        check(load().anc_mf_set_wait_ns(self._h, int(ns)))

    def pad(self, m: torch.Tensor) -> torch.Tensor:
        """[R, n] (R <= 64) -> [64, npad] f32 on the device, zero padded."""
        R, n = m.shape
        if R > REPLICAS or n != self.n:
            raise ValueError(f"magnetisations must be [R <= {REPLICAS}, {self.n}]")
        out = torch.zeros((REPLICAS, self.npad), dtype=torch.float32, device="cuda")
        out[:R, :n] = m.to(device="cuda", dtype=torch.float32)
        return out

    def __del__(self):
        lib = getattr(_lib, "_lib", None) if _lib is not None else None
        if getattr(self, "_h", None) and lib is not None and self._h.value:
            lib.anc_mf_destroy(self._h)
            self._h = C.c_void_p()


class _Relax(torch.autograd.Function):
    @staticmethod
    def forward(ctx, beta, q, u, w, mf: MeanField, m0, mprev):
        sched = torch.stack([beta, q, u, w]).to(device="cuda", dtype=torch.float32).contiguous()
        out, ck = mf.forward_raw(sched, m0.contiguous(), mprev.contiguous())
        ctx.mf = mf
        ctx.dtypes = (beta.dtype, q.dtype, u.dtype, w.dtype)
        ctx.save_for_backward(sched, ck)
        return out

    @staticmethod
    def backward(ctx, g):
        sched, ck = ctx.saved_tensors
        gs = ctx.mf.backward_raw(sched, ck, g.to(torch.float32).contiguous())
        tot = gs.double().sum(dim=2)       # per-replica partials summed in a fixed order
        return tuple(tot[:, k].to(ctx.dtypes[k]) for k in range(4)) + (None, None, None)


def relax(mf: MeanField, beta, q, u, w, m0: torch.Tensor, mprev: Optional[torch.Tensor] = None) -> torch.Tensor:
    """m_S [64, npad] of the relaxation from m0 ([64, npad]; mprev defaults to +1 on active slots, the golden model's
    initial s_prev). Differentiable in the per-step vectors beta, q, u, w ([S] each)."""
    if mprev is None:
        mprev = torch.zeros_like(m0)
        mprev[:, : mf.n] = 1.0
    return _Relax.apply(beta, q, u, w, mf, m0, mprev)


@dataclasses.dataclass
class SoftSchedule:
    """Five-parameter schedule family of the exact engine's tables (tables.hpp:14-40 with a linear q ramp):
    T_t = T0 exp(-rate t / (S-1)), q_t = q0 + q_slope t / (S-1), correction gain g applied as lambda (counted
    Onsager) or kappa (temperature-scaled) with the optional 0.7 S ramp."""

    S: int
    mode: str = "counted"      # "counted" | "tecT" | "none"
    ramp: bool = True

    def _ramp(self, dtype, device):
        S = self.S
        t = torch.arange(S, dtype=dtype, device=device)
        rden = max((S - 1) - 0.7 * S, 1.0)
        rf = torch.where(t >= 0.7 * S, (S - 1 - t) / rden, torch.ones_like(t)) if self.ramp else torch.ones_like(t)
        return t, rf

    def temperatures(self, theta: torch.Tensor) -> torch.Tensor:
        t, _ = self._ramp(theta.dtype, theta.device)
        return theta[0] * torch.exp(-theta[1] * t / max(self.S - 1, 1))

    def vectors(self, theta: torch.Tensor):
        """theta = [T0, rate, q0, q_slope, gain] -> per-step (beta, q, u, w), differentiable."""
        t, rf = self._ramp(theta.dtype, theta.device)
        T = self.temperatures(theta)
        beta = 1.0 / (2.0 * T)
        q = theta[2] + theta[3] * t / max(self.S - 1, 1)
        Tprev = torch.cat([T[:1], T[:-1]])
        first = (t > 0).to(theta.dtype)
        zero = torch.zeros_like(t)
        if self.mode == "counted":
            u, w = first * theta[4] * rf / (2.0 * Tprev), zero
        elif self.mode == "tecT":
            u, w = zero, first * theta[4] * Tprev * rf
        else:
            u, w = zero, zero
        return beta, q, u, w

    def tables(self, theta):
        """The exact engine's Tables (device) for theta; see table_arrays."""
        from .engine import Tables
        return Tables.from_arrays(**self.table_arrays(theta))

    def table_arrays(self, theta) -> dict:
        """The exact engine's integer tables for theta as host arrays (same rounding as the reference: llround of
        4T 2^16, q 2^16, lambda/(2 T_{t-1}) 2^24, kappa T_{t-1} 2^16)."""
        th = [float(x) for x in (theta.tolist() if isinstance(theta, torch.Tensor) else theta)]
        S = self.S
        t0, t1 = th[0], th[0] * math.exp(-th[1])
        den = S - 1 if S - 1 > 1 else 1
        T = [t0 * math.pow(t1 / t0, t / den) for t in range(S)]     # the reference's geometric form
        rden = max((S - 1) - 0.7 * S, 1.0)
        fourT = np.array([_llround(4.0 * T[t] * 65536.0) for t in range(S)], np.int32)
        q = np.array([_llround((th[2] + th[3] * t / max(S - 1, 1)) * 65536.0) for t in range(S)], np.int32)
        kcorr = np.zeros(S, np.int64)
        kconst = np.zeros(S, np.int32)
        for t in range(1, S):
            rf = (S - 1 - t) / rden if (self.ramp and t >= 0.7 * S) else 1.0
            if self.mode == "counted":
                kcorr[t] = _llround(th[4] * rf / (2.0 * T[t - 1]) * 16777216.0)
            elif self.mode == "tecT":
                kconst[t] = _llround(th[4] * T[t - 1] * rf * 65536.0)
        return dict(fourT=fourT, q=q, kcorr=kcorr, kconst=kconst)


def _llround(x: float) -> int:
    """C llround: halves away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def soft_cut(inst: Instance, m: torch.Tensor, J: Optional[torch.Tensor] = None,
             sumw: Optional[int] = None) -> torch.Tensor:
    """Cut of magnetisations m [R, n] by the golden model's formula (sumw + m^T J m / 2) / 2 (sca_ref.hpp:153
    without the integer truncation); equals the exact cut for m in {-1, +1}^n. Pass J (on m's device) and sumw to
    avoid recomputing them."""
    if J is None:
        J = torch.as_tensor(inst.to_dense(), dtype=m.dtype, device=m.device)
    if sumw is None:
        sumw = inst.stats()["sumw"]
    return (sumw + 0.5 * ((m @ J.to(m.dtype)) * m).sum(dim=1)) / 2.0


def initial_magnetisations(n: int, R: int, seed: int) -> torch.Tensor:
    """R seeded uniform +-1 starting points [R, n] (f32)."""
    g = torch.Generator().manual_seed(seed)
    return (torch.randint(0, 2, (R, n), generator=g) * 2 - 1).to(torch.float32)


def tune(inst: Instance, S: int = 200, R: int = 64, theta0=(30.0, math.log(6.0), 4.0, 0.0, 1.05), mode="counted",
         iters: int = 30, lr: float = 0.05, seed: int = 1, log=None):
    """Gradient ascent of the mean soft cut over theta = (T0, rate, q0, q_slope, gain) with Adam, the positive
    parameters (T0, rate) in log space. Returns (theta with the highest soft cut seen, history of (iteration, soft
    cut, theta)); Adam's steps are not monotone, so the last iterate need not be the best."""
    mf = MeanField(inst)
    sch = SoftSchedule(S=S, mode=mode)
    m0 = mf.pad(initial_magnetisations(inst.n, R, seed))
    J = torch.as_tensor(inst.to_dense(), dtype=torch.float32, device="cuda")
    sumw = inst.stats()["sumw"]
    raw = torch.tensor([math.log(theta0[0]), math.log(max(theta0[1], 1e-3)), theta0[2], theta0[3], theta0[4]],
                       dtype=torch.float64, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([raw], lr=lr)
    hist = []
    for it in range(iters):
        theta = torch.stack([raw[0].exp(), raw[1].exp(), raw[2], raw[3], raw[4]])
        beta, q, u, w = sch.vectors(theta)
        mS = relax(mf, beta, q, u, w, m0)
        cut = soft_cut(inst, mS[:R, : inst.n], J, sumw).mean()
        opt.zero_grad()
        (-cut).backward()
        opt.step()
        hist.append((it, cut.item(), [float(x) for x in theta.detach().tolist()]))
        if log:
            log(hist[-1])
    best = max(hist, key=lambda h: h[1])
    return torch.tensor(best[2], dtype=torch.float64, device="cuda"), hist


def judge(inst: Instance, S: int, thetas: dict, nchains: int = 1024, seed: int = 20261004, trial_offset: int = 0,
          targets: Optional[dict] = None, mode: str = "counted", engine: str = "auto") -> dict:
    """Judge schedules on the exact integer engine only: for each named theta (T0, rate, q0, q_slope, gain) the
    integer tables of SoftSchedule(S, mode).table_arrays run nchains anneals (the same trial ids for every schedule)
    and each named target cut t gives p = P(cut >= t) with its Wilson 95 % interval and the secondary TTS99
    t_batch ln(0.01) / (B ln(1 - p)) (the reference's estimators, analyze.py:15-47). targets defaults to
    {"median_first": the median cut of the first schedule}. Returns {name: {...}} plus the targets used."""
    from . import analyze
    from .engine import DeviceInstance, Tables, run
    dev = DeviceInstance(inst)
    sumw = inst.stats()["sumw"]
    cuts, times, kernels = {}, {}, {}
    for name, th in thetas.items():
        tb = Tables.from_arrays(**SoftSchedule(S=S, mode=mode).table_arrays(th))
        run(dev, tb, seed, 0xB0000000, min(nchains, 128), engine=engine)          # warm-up (untimed, other trials)
        r = run(dev, tb, seed, trial_offset, nchains, engine=engine)
        cuts[name], times[name], kernels[name] = r.cuts(sumw), r.device_ms, r.kernel
    first = next(iter(thetas))
    if targets is None:
        targets = {"median_first": int(np.median(cuts[first]))}
    out = {"targets": dict(targets), "S": S, "anneals": nchains, "engine_kernels": kernels}
    for name in thetas:
        c = cuts[name]
        th = thetas[name]
        rec = {"theta": [float(x) for x in (th.tolist() if isinstance(th, torch.Tensor) else th)],
               "mean_cut": float(c.mean()), "best_cut": int(c.max()), "ms_per_batch": times[name]}
        for tn, tv in targets.items():
            k = int((c >= tv).sum())
            p = k / nchains
            lo, hi = analyze.wilson(k, nchains)
            rec[tn] = {"p": p, "p_wilson95": [lo, hi], "successes": k,
                       "tts99_ms_secondary": analyze.tts99_secondary(p, nchains, times[name])}
        out[name] = rec
    return out


def main(argv=None) -> int:
    """Tune a schedule on the relaxation, then judge it against the starting schedule on the exact engine:

        python -m anechoic_b200.meanfield (--graph F | --gset F | --jint8 F) [--bias F] [--steps 200] [--iters 40]
                                          [--lr 0.01] [--mode counted|tecT|none] [--anneals 1024] [--seed S]
                                          [--t0 30 --rate 1.792 --q0 4 --q-slope 0 --gain 1.05]

    Prints one JSON line: the tuning history's first and best soft cut, the tuned theta (T0, rate, q0, q slope,
    gain) and its integer tables' judgement (anc engine, p at the starting schedule's median cut). --iters 1 runs a
    single forward and adjoint pass (as a profiler capture needs)."""
    import argparse
    import json
    from .instances import load, read_bias
    ap = argparse.ArgumentParser(prog="python -m anechoic_b200.meanfield")
    for k in ("--graph", "--gset", "--jint8"):
        ap.add_argument(k)
    ap.add_argument("--bias")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--iters", type=int, default=40)
    ap.add_argument("--lr", type=float, default=0.01)
    ap.add_argument("--mode", default="counted", choices=["counted", "tecT", "none"])
    ap.add_argument("--anneals", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=20261004)
    ap.add_argument("--t0", type=float, default=30.0)
    ap.add_argument("--rate", type=float, default=math.log(6.0))
    ap.add_argument("--q0", type=float, default=4.0)
    ap.add_argument("--q-slope", type=float, default=0.0)
    ap.add_argument("--gain", type=float, default=1.05)
    ap.add_argument("--no-judge", action="store_true")
    a = ap.parse_args(argv)
    kind = next((k for k in ("graph", "gset", "jint8") if getattr(a, k)), None)
    if kind is None:
        ap.error("one of --graph, --gset, --jint8 is required")
    inst = load(kind, getattr(a, kind))
    if a.bias:
        inst.bias = read_bias(a.bias, inst.n)
    theta0 = (a.t0, a.rate, a.q0, a.q_slope, a.gain)
    tuned, hist = tune(inst, S=a.steps, theta0=theta0, mode=a.mode, iters=a.iters, lr=a.lr)
    best = max(hist, key=lambda h: h[1])
    line = {"n": inst.n, "steps": a.steps, "iters": len(hist), "soft_cut_first": hist[0][1], "soft_cut_best": best[1],
            "theta0": list(theta0), "theta_tuned": best[2]}
    if not a.no_judge:
        line["judgement"] = judge(inst, a.steps, {"start": torch.tensor(theta0, dtype=torch.float64),
                                                  "tuned": tuned.cpu()}, nchains=a.anneals, seed=a.seed,
                                  mode=a.mode)
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
