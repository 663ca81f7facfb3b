"""TEST INFRASTRUCTURE AND CPU BASELINE ONLY: this project's numba restatements of the reference's two float research
models of the SCA engine, timed as the "numba SCA" CPU baseline. They are statistical models (their own RNGs, float
thresholds), not bit-exact checkers; bench.py's CPU-baseline leg runs them on the host cores beside the exact golden
model. The product never imports this module.

fused_int_model  restates research/optimum_mitigation_20261007/sca_fast.py:102-165 (run_steps): integer spins and
                 fields, one anneal per thread (numba prange), a splitmix64 stream per anneal from which a uniform
                 is drawn only for slots inside the linear band, z in float64, and the field update as the doubled
                 coupling rows of the flipped spins.
sequential_model restates research/gset_20261007/engine.py:99-188 (run / _step): float32 spins and fields, one
                 uniform per slot and step (a numpy float32 block per step, as abl.run draws it), the counted
                 correction evaluated in float64 (field h - lambda c_prev s_prev), CSR row scatter of the flipped
                 spins, and the anneals advanced one after another in a single thread.
Both use the reference's schedule formulas: T_t = T0 (T1 / T0)^(t / (S - 1)), counted Onsager coefficient
lambda ramp(t) / (2 T_{t-1}) with the 0.7 S ramp (sca_fast.py:56-87).
"""
from __future__ import annotations

import math

import numpy as np
import numba as nb

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_MIX1 = np.uint64(0xBF58476D1CE4E5B9)
_MIX2 = np.uint64(0x94D049BB133111EB)


def ramp_factors(S: int, ramp: bool, start: float = 0.7) -> np.ndarray:
    t = np.arange(S, dtype=np.float64)
    if not ramp:
        return np.ones(S)
    return np.where(t < start * S, 1.0, (S - 1 - t) / max(1.0, S - 1 - start * S))


def schedule(S: int, T0: float, T1: float, q: float, lam: float, ramp: bool):
    """Per-step (T, q, a, b) of the counted-Onsager family: a_t = lam ramp(t) / (2 T_{t-1}) for t >= 1."""
    T = T0 * (T1 / T0) ** (np.arange(S) / max(1, S - 1))
    a = np.zeros(S)
    a[1:] = lam * ramp_factors(S, ramp)[1:] / (2.0 * T[:-1])
    return T.astype(np.float64), np.full(S, float(q)), a, np.zeros(S)


@nb.njit(inline="always")
def _splitmix(x):
    x = x + _GOLDEN
    z = x
    z = (z ^ (z >> np.uint64(30))) * _MIX1
    z = (z ^ (z >> np.uint64(27))) * _MIX2
    return x, z ^ (z >> np.uint64(31))


@nb.njit(parallel=True, cache=True)
def _fused_int(J2, s, sp, h, rng, flips, T, q, a, b):
    B, N = s.shape
    S = T.shape[0]
    for r in nb.prange(B):
        x = rng[r]
        flipped = np.empty(N, np.int32)
        nl = 0
        fl = 0
        for t in range(S):
            fourT = 4.0 * T[t]
            twoT = 2.0 * T[t]
            corr = a[t] * nl + b[t]
            nf = 0
            cnt = 0
            for i in range(N):
                shi = np.int64(s[r, i]) * np.int64(h[r, i])
                z = shi + q[t] - corr if s[r, i] == sp[r, i] else shi + q[t] + corr
                if z <= -twoT:
                    flipped[nf] = i
                    nf += 1
                elif z < twoT:
                    cnt += 1
                    x, v = _splitmix(x)
                    u = np.float64(v >> np.uint64(40)) * (1.0 / 16777216.0)
                    if z / fourT + 0.5 < u:
                        flipped[nf] = i
                        nf += 1
            for i in range(N):
                sp[r, i] = s[r, i]
            for k in range(nf):
                i = flipped[k]
                s[r, i] = -s[r, i]
                row = J2[i]
                if s[r, i] > 0:
                    for y in range(N):
                        h[r, y] += row[y]
                else:
                    for y in range(N):
                        h[r, y] -= row[y]
            fl += nf
            nl = cnt
        rng[r] = x
        flips[r] = fl


def fused_int_model(J: np.ndarray, B: int, seed: int, sched):
    """B anneals of the integer fused model (one per thread). Returns (spins int8 [B, N], flips)."""
    N = J.shape[0]
    g = np.random.default_rng(seed)
    s = np.where(g.random((B, N)) < 0.5, -1, 1).astype(np.int8)
    sp = s.copy()
    h = (s.astype(np.int32) @ J.astype(np.int32)).astype(np.int16)
    rng = g.integers(0, 2 ** 63 - 1, size=B, dtype=np.int64).astype(np.uint64)
    flips = np.zeros(B, np.int64)
    J2 = (2 * J).astype(np.int8)
    T, q, a, b = sched
    _fused_int(J2, s, sp, h, rng, flips, T, q, a, b)
    return s, flips


@nb.njit(cache=True)
def _seq_step(onsager, s, h, sp, u, Tt, c64, cprev, cnt, flips, indptr, indices, data, qv, flipbuf):
    B, N = s.shape
    d4 = 4.0 * Tt
    lo, hi = -2.0 * Tt, 2.0 * Tt
    d4f = np.float32(d4)
    for r in range(B):
        nlin = 0
        nfl = 0
        cb = c64 * cprev[r]
        for i in range(N):
            if onsager:
                z = np.float64(s[r, i]) * (np.float64(h[r, i]) - cb * np.float64(sp[r, i])) + qv
                x = min(max(z / d4 + 0.5, 0.0), 1.0)
                f = x < np.float64(u[r, i])
                if z > lo and z < hi:
                    nlin += 1
            else:
                z32 = s[r, i] * h[r, i] + np.float32(qv)
                x32 = min(max(z32 / d4f + np.float32(0.5), np.float32(0.0)), np.float32(1.0))
                f = x32 < u[r, i]
                if z32 > np.float32(lo) and z32 < np.float32(hi):
                    nlin += 1
            if f:
                flipbuf[nfl] = i
                nfl += 1
        cnt[r] = nlin
        flips[r] += nfl
        for i in range(N):
            sp[r, i] = s[r, i]
        for k in range(nfl):
            i = flipbuf[k]
            d = np.float32(-2.0) * s[r, i]
            s[r, i] = s[r, i] + d
            for e in range(indptr[i], indptr[i + 1]):
                h[r, indices[e]] += d * data[e]


def sequential_model(J: np.ndarray, B: int, seed: int, S: int, T0: float, T1: float, q: float, lam: float,
                     ramp: bool):
    """B anneals of the sequential float32 model, advanced together one step at a time in one thread. Returns
    (spins float32 [B, N], flips)."""
    N = J.shape[0]
    rows, cols = np.nonzero(J)
    indptr = np.zeros(N + 1, np.int64)
    np.add.at(indptr, rows + 1, 1)
    indptr = np.cumsum(indptr)
    indices = cols.astype(np.int64)
    data = J[rows, cols].astype(np.float32)
    g = np.random.default_rng(seed)
    s = np.where(g.random((B, N)) < 0.5, -1.0, 1.0).astype(np.float32)
    h = (s @ J.astype(np.float32)).astype(np.float32)
    sp = np.zeros_like(s)
    cprev = np.zeros(B)
    cnt = np.zeros(B, np.int64)
    flips = np.zeros(B)
    flipbuf = np.zeros(N, np.int64)
    T = T0 * (T1 / T0) ** (np.arange(S) / max(1, S - 1))
    rf = ramp_factors(S, ramp)
    for t in range(S):
        u = g.random(s.shape, dtype=np.float32)
        onsager = t > 0 and lam > 0
        c64 = lam * rf[t] if onsager else 0.0
        _seq_step(onsager, s, h, sp, u, float(T[t]), c64, cprev, cnt, flips, indptr, indices, data, float(q), flipbuf)
        if lam > 0:
            cprev = cnt / (2.0 * T[t])
    return s, flips


def cut_of(J: np.ndarray, s: np.ndarray) -> np.ndarray:
    """Max-Cut value of each row of s (+-1) with weights w = -J: (sum_{i<j} w_ij (1 - s_i s_j)) / 2."""
    Jf = J.astype(np.float64)
    sf = s.astype(np.float64)
    sumw = -np.triu(Jf, 1).sum()
    return np.rint((sumw + 0.5 * ((sf @ Jf) * sf).sum(axis=1)) / 2.0).astype(np.int64)


def time_models(J: np.ndarray, S: int, T0: float, T1: float, q: float, lam: float, ramp: bool, cores: int,
                budget_s: float = 6.0) -> dict:
    """Anneals/s of both models on the host cores (numba compile excluded: one tiny call first). The fused model runs
    `cores` anneals per round in parallel; the sequential model runs one anneal per round in a single thread. Each is
    timed over whole rounds until about budget_s seconds have passed."""
    nb.set_num_threads(max(1, min(cores, nb.config.NUMBA_NUM_THREADS)))
    threads = nb.get_num_threads()
    sched = schedule(S, T0, T1, q, lam, ramp)
    small = schedule(4, T0, T1, q, lam, ramp)
    fused_int_model(J, threads, 1, small)                   # compile
    sequential_model(J, 1, 1, 4, T0, T1, q, lam, ramp)      # compile
    out = {}
    rounds, t0 = 0, __import__("time").perf_counter()
    cuts = []
    while True:
        s, _ = fused_int_model(J, threads, 100 + rounds, sched)
        cuts.append(cut_of(J, s))
        rounds += 1
        dt = __import__("time").perf_counter() - t0
        if dt >= budget_s or rounds >= 64:
            break
    c = np.concatenate(cuts)
    out["fused_int"] = {"value": rounds * threads / dt, "unit": "anneals/s", "cores": threads, "kind": "port",
                        "sample": f"{rounds * threads} anneals x S={S} in {dt:.1f} s ({threads} threads, one anneal "
                                  f"per thread)",
                        "mean_cut": float(c.mean()),
                        "model": "research/optimum_mitigation_20261007/sca_fast.py:102 run_steps (numba restatement)"}
    rounds, t0 = 0, __import__("time").perf_counter()
    cuts = []
    while True:
        s, _ = sequential_model(J, 1, 200 + rounds, S, T0, T1, q, lam, ramp)
        cuts.append(cut_of(J, s))
        rounds += 1
        dt = __import__("time").perf_counter() - t0
        if dt >= budget_s or rounds >= 64:
            break
    c = np.concatenate(cuts)
    out["sequential"] = {"value": rounds / dt, "unit": "anneals/s", "cores": 1, "kind": "port",
                         "sample": f"{rounds} anneals x S={S} in {dt:.1f} s (1 thread)",
                         "mean_cut": float(c.mean()),
                         "model": "research/gset_20261007/engine.py:159 run (numba restatement)"}
    return out
