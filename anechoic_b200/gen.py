"""Instance generators of the reference's bias study (gpu/multibit_bias_20261008/src/gen_ising.cpp), restated:
the same seeded splitmix64 streams, the same encodings, the same output files (PREFIX.jint8 SCAJINT8 couplings,
PREFIX.bias SCABIAS1 biases, PREFIX.json metadata; gp also PREFIX.edges).

Model: H(s) = -sum_{i<j} J_ij s_i s_j - sum_i b_i s_i, s in {-1, +1}, x = (1 + s) / 2.

    python -m anechoic_b200.gen random --n N --kbits K --pzero P --bmax B [--pbig Q --bsmall b] --seed S --out PREFIX
    python -m anechoic_b200.gen zero --n N --out FILE.bias
    python -m anechoic_b200.gen gp --n N --deg D --k K --A a --B b --seed S --out PREFIX [--brute 1]
    python -m anechoic_b200.gen tsp --n CITIES --wmax W --A a --B b --seed S --out PREFIX [--brute 1]
    python -m anechoic_b200.gen brute --jint8 F [--bias F]

gp (graph partitioning, Lucas 2014, unbalanced sizes; gen_ising.cpp:145-197): a random D-regular simple graph from
the pairing model with rejection, minimise the cut subject to |{x = 1}| = K:
f(x) = b cut(x) + a (sum x - K)^2, J_ij = -a + b [ij in E], b_i = a (2K - n), H = 2 f + C.
tsp (Lucas 2014; gen_ising.cpp:198-280): city 0 fixed at position 0, spin (v-1)(n-1) + (p-1) = city v at position p
(v, p in 1..n-1), symmetric distances uniform in 1..W; f = a sum_v (1 - sum_p x_vp)^2 + a sum_p (1 - sum_v x_vp)^2
+ b * tour length, J_ij = -Q_ij, b_i = -(2 c_i + sum_j Q_ij), H = 4 f + C.
Both check H = sigma f + C on 200 random states; --brute 1 (n <= 30) also enumerates every spin state for the Ising
minimum and checks it against a direct enumeration of the problem (all K-subsets, all tours).
"""
from __future__ import annotations

import itertools
import json
import sys
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import instances as I

M64 = (1 << 64) - 1
NP_MAX = 2048


class SplitMix:
    """splitmix64 (the generator's own stream, gen_ising.cpp:24-29)."""

    def __init__(self, seed: int):
        self.x = seed & M64

    def next(self) -> int:
        self.x = (self.x + 0x9E3779B97F4A7C15) & M64
        z = self.x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)


def ising_energy(J: np.ndarray, b: np.ndarray, S: np.ndarray) -> np.ndarray:
    """H of each row of S (+-1 states): -sum_{i<j} J_ij s_i s_j - sum_i b_i s_i, int64."""
    S = np.atleast_2d(np.asarray(S, np.int64))
    Jl = J.astype(np.int64)
    return -(((S @ Jl) * S).sum(axis=1) // 2) - S @ b.astype(np.int64)


def _check_relation(J, b, f_of, sigma: int, C: int, seed: int, what: str):
    st = SplitMix(seed)
    n = len(b)
    S = np.array([[1 if (st.next() & 1) else -1 for _ in range(n)] for _ in range(200)], np.int64)
    H = ising_energy(J, b, S)
    F = np.array([f_of(s) for s in S], np.int64)
    if np.any(H != sigma * F + C):
        raise RuntimeError(f"{what}: H != {sigma}f + C on random states")


def brute_force(J: np.ndarray, b: np.ndarray, keep: int = 64) -> Tuple[int, int, List[np.ndarray]]:
    """Exhaustive Ising minimum over all 2^n states (n <= 30): (emin, number of ground states, up to `keep` of them
    in increasing order of their bit pattern, bit i = [s_i = +1])."""
    n = len(b)
    if n > 30:
        raise ValueError("brute force limited to n <= 30")
    emin, count, gs = None, 0, []
    chunk = 1 << min(n, 16)
    bits = (np.arange(n, dtype=np.int64))
    for start in range(0, 1 << n, chunk):
        m = np.arange(start, min(start + chunk, 1 << n), dtype=np.int64)
        S = np.where((m[:, None] >> bits) & 1, 1, -1)
        E = ising_energy(J, b, S)
        lo = int(E.min())
        if emin is None or lo < emin:
            emin, count, gs = lo, 0, []
        if lo == emin:
            hit = np.nonzero(E == emin)[0]
            count += len(hit)
            for k in hit[: max(0, keep - len(gs))]:
                gs.append(S[k])
    return emin, count, gs


def _meta_text(meta: Dict) -> str:
    """Compact JSON with C++ stream number formatting (doubles as %g), as the reference generator prints."""
    def fmt(v):
        if isinstance(v, bool):
            return "true" if v else "false"
        if isinstance(v, float):
            return format(v, "g")
        if isinstance(v, dict):
            return "{" + ",".join(f'"{k}":{fmt(x)}' for k, x in v.items()) + "}"
        if isinstance(v, (list, tuple)):
            return "[" + ",".join(fmt(x) for x in v) + "]"
        if isinstance(v, str):
            return json.dumps(v)
        return str(int(v))
    return fmt(meta)


def _instance(J: np.ndarray, b: np.ndarray, name: str) -> I.Instance:
    if np.any(np.abs(J) > 127):
        raise ValueError("coupling outside int8")
    inst = I.Instance(n=len(b), dense=J.astype(np.int8), bias=b.astype(np.int32), name=name)
    inst.validate()
    return inst


def random_instance(n: int, kbits: int, seed: int, pzero: float = 0.0, bmax: int = 0, pbig: float = 1.0,
                    bsmall: int = 0) -> Tuple[I.Instance, Dict]:
    """gen_ising random (gen_ising.cpp:118-143): J from the coupling stream, b uniform in [-bmax, bmax] with
    probability pbig, otherwise in [-bsmall, bsmall]."""
    if kbits < 2 or kbits > 8 or n < 1 or n > NP_MAX:
        raise ValueError("random: 2 <= K <= 8, 1 <= n <= 2048")
    base = I.random_kbit(n, kbits, seed, pzero=pzero, bmax=bmax if pbig >= 1.0 else 0)
    b = base.bias if base.bias is not None else np.zeros(n, np.int32)
    if pbig < 1.0:
        sb = SplitMix(seed ^ 0x5B1A5B1A5B1A5B1A)
        b = np.zeros(n, np.int32)
        for i in range(n):
            big = (sb.next() >> 11) * 2.0 ** -53 < pbig
            bm = bmax if big else bsmall
            b[i] = (sb.next() % (2 * bm + 1)) - bm if bm > 0 else 0
    inst = _instance(base.dense, b, f"random_n{n}_k{kbits}_s{seed}")
    st = inst.stats()
    meta = {"type": "random", "N": n, "kbits": kbits, "pzero": float(pzero), "bmax_param": bmax, "pbig": float(pbig),
            "bsmall": bsmall, "seed": seed, "maxabs": st["maxabs"], "hmax": st["hmax"],
            "bmax": int(np.abs(b.astype(np.int64)).max()) if n else 0, "sumw": st["sumw"]}
    return inst, meta


def graph_partitioning(n: int, k: int, deg: int = 3, A: int = 1, B: int = 1, seed: int = 1,
                       brute: bool = False) -> Tuple[I.Instance, Dict, List[Tuple[int, int]]]:
    """gen_ising gp. Returns the instance, its metadata and the sorted edge list."""
    if n < 4 or n > NP_MAX or k < 1 or k >= n or (n * deg) % 2:
        raise ValueError("gp: bad arguments")
    st = SplitMix(seed ^ 0x6A09E667F3BCC908)
    attempts = 0
    while True:
        attempts += 1
        stubs = [v for v in range(n) for _ in range(deg)]
        for i in range(len(stubs) - 1, 0, -1):
            j = st.next() % (i + 1)
            stubs[i], stubs[j] = stubs[j], stubs[i]
        E, ok = set(), True
        for t in range(0, len(stubs), 2):
            u, v = sorted((stubs[t], stubs[t + 1]))
            if u == v or (u, v) in E:
                ok = False
                break
            E.add((u, v))
        if ok:
            break
        if attempts > 100000:
            raise RuntimeError("no simple regular graph")
    edges = sorted(E)
    adj = np.zeros((n, n), np.int64)
    if edges:
        e = np.array(edges)
        adj[e[:, 0], e[:, 1]] = 1
        adj[e[:, 1], e[:, 0]] = 1
    J = -A + B * adj
    np.fill_diagonal(J, 0)
    b = np.full(n, A * (2 * k - n), np.int64)
    ea = np.array(edges, np.int64)

    def f_parts(s):
        x = s > 0
        cut = int(np.count_nonzero(x[ea[:, 0]] != x[ea[:, 1]]))
        sx = int(x.sum())
        return B * cut + A * (sx - k) ** 2, cut, sx

    inst = _instance(J, b, f"gp_n{n}_d{deg}_k{k}_s{seed}")
    C = int(ising_energy(J, b, -np.ones(n, np.int64))[0]) - 2 * f_parts(-np.ones(n, np.int64))[0]
    _check_relation(J, b, lambda s: f_parts(s)[0], 2, C, seed ^ 0x1234, "gp")
    st_ = inst.stats()
    meta = {"type": "graph_partitioning", "N": n, "deg": deg, "k": k, "A": A, "B": B, "seed": seed,
            "edges": len(edges), "sigma": 2, "C": C,
            "relation": "H = 2 f + C, f = B*cut + A*(sum x - k)^2, x_i = (1+s_i)/2",
            "maxabs": st_["maxabs"], "hmax": st_["hmax"], "bmax": abs(A * (2 * k - n))}
    if brute:
        if n > 30:
            raise ValueError("gp brute force limited to n <= 30")
        emin, count, gs = brute_force(J, b)
        best, nbest = None, 0
        for sub in itertools.combinations(range(n), k):
            x = np.zeros(n, bool)
            x[list(sub)] = True
            cut = int(np.count_nonzero(x[ea[:, 0]] != x[ea[:, 1]]))
            if best is None or cut < best:
                best, nbest = cut, 0
            nbest += cut == best
        feas = bool(all(f_parts(g)[2] == k and f_parts(g)[1] == best for g in gs))
        ok = bool(emin == 2 * B * best + C and feas and count == nbest)
        meta["brute"] = {"ising_emin": emin, "ising_ground_states": count, "direct_min_cut": best,
                         "direct_optima": nbest, "emin_expected": 2 * B * best + C,
                         "ground_states_feasible_optimal": feas, "consistent": ok}
        if not ok:
            raise RuntimeError("gp brute-force check failed")
    return inst, meta, edges


def tsp(cities: int, wmax: int = 2, A: int = 1, B: int = 1, seed: int = 1,
        brute: bool = False) -> Tuple[I.Instance, Dict]:
    """gen_ising tsp."""
    n = cities
    if n < 3 or (n - 1) * (n - 1) > NP_MAX or wmax < 1:
        raise ValueError("tsp: bad arguments")
    m = n - 1
    nv = m * m
    st = SplitMix(seed ^ 0x3C6EF372FE94F82B)
    W = np.zeros((n, n), np.int64)
    for u in range(n):
        for v in range(u + 1, n):
            W[u, v] = W[v, u] = 1 + st.next() % wmax

    def idx(v, p):
        return (v - 1) * m + (p - 1)

    Q = np.zeros((nv, nv), np.int64)
    c = np.zeros(nv, np.int64)
    c0 = 0

    def addQ(i, j, val):
        if i > j:
            i, j = j, i
        Q[i, j] += val

    for v in range(1, m + 1):      # city v visited once, position v filled once
        c0 += 2 * A
        for p in range(1, m + 1):
            c[idx(v, p)] -= A
            c[idx(p, v)] -= A
            for p2 in range(p + 1, m + 1):
                addQ(idx(v, p), idx(v, p2), 2 * A)
                addQ(idx(p, v), idx(p2, v), 2 * A)
    for p in range(1, m):
        for u in range(1, m + 1):
            for v in range(1, m + 1):
                if u != v:
                    addQ(idx(u, p), idx(v, p + 1), B * W[u, v])
    for v in range(1, m + 1):
        c[idx(v, 1)] += B * W[0, v]
        c[idx(v, m)] += B * W[v, 0]
    Qs = Q + Q.T                    # Q has no diagonal
    J = -Qs
    b = -(2 * c + Qs.sum(axis=1))
    if np.any(np.abs(b) > 32767):
        raise ValueError("tsp bias outside 16 bits")

    def f_of(s):
        x = (np.asarray(s) > 0).astype(np.int64)
        return int(c0 + c @ x + x @ np.triu(Q, 1) @ x)

    inst = _instance(J, b, f"tsp_c{n}_w{wmax}_s{seed}")
    C = int(ising_energy(J, b, -np.ones(nv, np.int64))[0]) - 4 * f_of(-np.ones(nv, np.int64))
    _check_relation(J, b, f_of, 4, C, seed ^ 0x777, "tsp")
    st_ = inst.stats()
    meta = {"type": "tsp", "cities": n, "N": nv, "wmax": wmax, "A": A, "B": B, "seed": seed, "sigma": 4, "C": C,
            "relation": "H = 4 f + C; valid tour: H = 4*B*length + C; spin (v-1)(n-1)+(p-1) = city v at position p; "
                        "city 0 at position 0",
            "maxabs": st_["maxabs"], "hmax": st_["hmax"], "bmax": int(np.abs(b).max()),
            "W": [[int(w) for w in row] for row in W]}
    if brute:
        if nv > 30:
            raise ValueError("tsp brute force limited to (n-1)^2 <= 30")
        emin, count, gs = brute_force(J, b)
        best, nbest = None, 0
        for perm in itertools.permutations(range(1, m + 1)):
            L = W[0, perm[0]] + W[perm[-1], 0] + sum(W[perm[p], perm[p + 1]] for p in range(m - 1))
            if best is None or L < best:
                best, nbest = int(L), 0
            nbest += int(L == best)
        all_opt = bool(all(tour_length(g, W) == best for g in gs))
        ok = bool(emin == 4 * B * best + C and all_opt and count == nbest)
        meta["brute"] = {"ising_emin": emin, "ising_ground_states": count, "direct_min_length": best,
                         "direct_optimal_tours": nbest, "emin_expected": 4 * B * best + C,
                         "ground_states_valid_optimal": all_opt, "consistent": ok}
        if not ok:
            raise RuntimeError("tsp brute-force check failed")
    return inst, meta


def tour_length(s, W: np.ndarray) -> int:
    """Tour length of a TSP spin state (city 0 at position 0), or -1 if the state is not a permutation."""
    n = W.shape[0]
    m = n - 1
    x = (np.asarray(s) > 0).reshape(m, m)          # [v - 1][p - 1]
    if not (np.all(x.sum(axis=0) == 1) and np.all(x.sum(axis=1) == 1)):
        return -1
    at = [int(np.nonzero(x[:, p])[0][0]) + 1 for p in range(m)]
    return int(W[0, at[0]] + W[at[-1], 0] + sum(W[at[p], at[p + 1]] for p in range(m - 1)))


def write(inst: I.Instance, meta: Dict, prefix: str, edges: Optional[List[Tuple[int, int]]] = None) -> str:
    """PREFIX.jint8, PREFIX.bias, PREFIX.json (and PREFIX.edges); returns the metadata text."""
    I.write_jint8(inst, prefix + ".jint8")
    I.write_bias(inst.bias if inst.bias is not None else np.zeros(inst.n, np.int32), prefix + ".bias")
    text = _meta_text(meta)
    with open(prefix + ".json", "w") as f:
        f.write(text + "\n")
    if edges is not None:
        with open(prefix + ".edges", "w") as f:
            f.writelines(f"{u} {v}\n" for u, v in edges)
    return text


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        if not argv:
            raise ValueError("usage: gen random|zero|gp|tsp|brute ...")
        cmd = argv[0]
        o = dict(out="", jint8="", bias="", n=0, kbits=2, deg=3, k=0, wmax=2, brute=0, pzero=0.0, bmax=0, A=1, B=1,
                 seed=1, pbig=1.0, bsmall=0)
        conv = dict(out=str, jint8=str, bias=str, n=int, kbits=int, deg=int, k=int, wmax=int, brute=int,
                    pzero=float, bmax=int, A=int, B=int, seed=int, pbig=float, bsmall=int)
        a = 1
        while a < len(argv):
            key = argv[a]
            if not key.startswith("--") or key[2:] not in conv:
                raise ValueError("unknown argument " + key)
            if a + 1 >= len(argv):
                raise ValueError("missing value for " + key)
            o[key[2:]] = conv[key[2:]](argv[a + 1])
            a += 2
        if cmd == "zero":
            if not o["out"] or o["n"] < 1 or o["n"] > NP_MAX:
                raise ValueError("zero: --n, --out")
            I.write_bias(np.zeros(o["n"], np.int32), o["out"])
            print(_meta_text({"wrote": o["out"], "N": o["n"]}))
            return 0
        if cmd == "brute":
            inst = I.read_jint8(o["jint8"])
            b = I.read_bias(o["bias"], inst.n) if o["bias"] else np.zeros(inst.n, np.int32)
            emin, count, _ = brute_force(inst.dense, b)
            print(_meta_text({"N": inst.n, "emin": emin, "ground_states": count}))
            return 0
        if not o["out"]:
            raise ValueError(cmd + ": --out required")
        edges = None
        if cmd == "random":
            inst, meta = random_instance(o["n"], o["kbits"], o["seed"], o["pzero"], o["bmax"], o["pbig"], o["bsmall"])
        elif cmd == "gp":
            inst, meta, edges = graph_partitioning(o["n"], o["k"], o["deg"], o["A"], o["B"], o["seed"], bool(o["brute"]))
        elif cmd == "tsp":
            inst, meta = tsp(o["n"], o["wmax"], o["A"], o["B"], o["seed"], bool(o["brute"]))
        else:
            raise ValueError("unknown command " + cmd)
        print(write(inst, meta, o["out"], edges))
        return 0
    except (ValueError, RuntimeError, OSError) as e:
        print("FAIL: " + str(e), file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
