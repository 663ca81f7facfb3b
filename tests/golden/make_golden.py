"""Generate the golden fixtures in this directory from the REFERENCE's own golden model.

The reference golden model (sca::run_trial, sca::run_trial_bias, v80host::build_tables, mb::tables; reference files
gpu/multibit_bias_20261008/src/{sca_ref.hpp,sca_ref_bias.hpp,tables.hpp,mb_common.hpp}) is compiled unmodified by
oracle/Makefile into oracle/_ref/libscaref.so with -DSCA_LANES=256, and called here through oracle/oracle.py.
Run from the repository root where the reference tree is available:

    make -C oracle && python tests/golden/make_golden.py

Instances come from this package's seeded generators; each fixture records the sha256 of its coupling matrix so the
generators stay pinned too.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from anechoic_b200 import instances as I  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

SEED = 20261004

# (name, schedule kwargs for v80host::build_tables)
PM1_SCHEDULES = [
    ("onsager", dict(S=300, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True)),
    ("tecT", dict(S=300, t0=30.0, t1=5.0, q=4.0, kappa=2.0, ramp=True)),
    ("plain", dict(S=300, t0=30.0, t1=5.0, q=4.0)),
    ("tec", dict(S=300, t0=30.0, t1=5.0, q=8.0, jv=-4.0)),
]

TABLE_CASES = [
    dict(S=1000, lam=1.05, ramp=True), dict(S=560), dict(S=300, q=8.0, jv=-4.0), dict(S=760, kappa=2.0, ramp=True),
    dict(S=120, t0=15.0, q=8.0, kappa=2.0, ramp=True), dict(S=960, lam=1.05, ramp=True), dict(S=7, lam=0.4, ramp=True),
    dict(S=2, lam=1.0, ramp=True), dict(S=1, lam=1.0), dict(S=5000, t0=200.0, t1=20.0, q=40.0, kappa=1.5, ramp=True),
]
MB_TABLE_CASES = [dict(S=500, lam=0.9, ramp=True, scale=0.37), dict(S=333, kappa=2.1, ramp=True, scale=1.7)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def tables_npz(prefix: str, tb: dict, out: dict):
    for k, v in tb.items():
        out[f"{prefix}{k}"] = v


def main():
    R = Reference()
    # 1. tables
    out = {}
    for k, c in enumerate(TABLE_CASES):
        tables_npz(f"c{k}_", R.build_tables(**c), out)
    for k, c in enumerate(MB_TABLE_CASES):
        tables_npz(f"mb{k}_", R.mb_tables(**c), out)
    np.savez_compressed(os.path.join(HERE, "tables.npz"), **out)

    # 2. +-1 complete graph, N = 2000: every mode, trials 0..3, with the full n_lin trace
    inst = I.complete_pm1(2000, SEED)
    st = inst.stats()
    out = dict(J_sha256=np.array(sha(inst.dense)), sumw=np.array(st["sumw"]))
    for name, sc in PM1_SCHEDULES:
        tb = R.build_tables(**sc)
        for trial in range(4):
            r = R.run_trial(inst.dense, st["sumw"], tb, SEED, trial)
            rb = R.run_trial_bias(2000, inst.dense, None, tb, SEED, trial)
            assert np.array_equal(r["spins"], rb["spins"]) and np.array_equal(r["nlin"], rb["nlin"])
            out[f"{name}_{trial}_spins"] = r["spins"]
            out[f"{name}_{trial}_cut"] = np.array(r["cut"])
            out[f"{name}_{trial}_sum_sh"] = np.array(rb["sum_sh"])
            out[f"{name}_{trial}_flips"] = np.array(r["flips"])
            out[f"{name}_{trial}_nlin"] = r["nlin"]
    np.savez_compressed(os.path.join(HERE, "pm1_n2000.npz"), **out)

    # 3. K = 4 couplings with bias, n = 800 (the shape of the reference's test_ref_bias.cpp part 2)
    k4 = I.random_kbit(800, 4, 7, pzero=1.0 / 15.0, bmax=300)
    tb = R.build_tables(S=200, t0=200.0, t1=20.0, q=40.0, lam=0.6, ramp=True)
    out = dict(J_sha256=np.array(sha(k4.dense)), bias_sha256=np.array(sha(k4.bias)))
    for trial in range(4):
        r = R.run_trial_bias(800, k4.dense, k4.bias, tb, 99, trial)
        for k in ("spins", "nlin"):
            out[f"t{trial}_{k}"] = r[k]
        for k in ("sum_sh", "sum_bs", "flips"):
            out[f"t{trial}_{k}"] = np.array(r[k])
    np.savez_compressed(os.path.join(HERE, "k4bias_n800.npz"), **out)

    # 4. ragged sizes with ternary couplings and bias (padding slots, partial words, n = 1)
    out = {}
    tb = R.build_tables(S=64, t0=3.0, t1=0.5, q=1.0, lam=0.5, ramp=True)
    for n in (1, 17, 257, 1000, 2048):
        g = I.random_kbit(n, 2, 5 + n, pzero=0.3, bmax=3) if n > 1 else I.Instance(
            n=1, dense=np.zeros((1, 1), np.int8), bias=np.array([3], np.int32))
        out[f"n{n}_J_sha256"] = np.array(sha(g.dense))
        for trial in range(2):
            r = R.run_trial_bias(n, g.dense, g.bias, tb, 5, trial)
            for k in ("spins", "nlin"):
                out[f"n{n}_t{trial}_{k}"] = r[k]
            for k in ("sum_sh", "sum_bs", "flips"):
                out[f"n{n}_t{trial}_{k}"] = np.array(r[k])
    np.savez_compressed(os.path.join(HERE, "ragged_k2.npz"), **out)

    # 5. a sparse +-1 graph with bias (G-set-shaped class), via its dense form
    sp = I.random_graph(800, 4690, True, 11, bmax=2)
    d = sp.to_dense()
    tb = R.build_tables(S=250, t0=6.0, t1=1.0, q=2.0, kappa=2.0, ramp=True)
    out = dict(J_sha256=np.array(sha(d)), bias_sha256=np.array(sha(sp.bias)))
    for trial in range(3):
        r = R.run_trial_bias(800, d, sp.bias, tb, SEED, 1000 + trial)
        for k in ("spins", "nlin"):
            out[f"t{trial}_{k}"] = r[k]
        for k in ("sum_sh", "sum_bs", "flips"):
            out[f"t{trial}_{k}"] = np.array(r[k])
    np.savez_compressed(os.path.join(HERE, "sparse_n800.npz"), **out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
