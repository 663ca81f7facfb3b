"""CPU: pin the C restatement of the golden model against fixtures generated by the reference's own golden model
(tests/golden/make_golden.py), and pin the instance generators by hash."""
import hashlib
import os

import numpy as np
import pytest

from anechoic_b200 import instances as I
from tests.conftest import GOLDEN
from tests.golden.make_golden import MB_TABLE_CASES, PM1_SCHEDULES, SEED, TABLE_CASES


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_tables_match_reference(oracle):
    g = _load("tables.npz")
    for k, c in enumerate(TABLE_CASES):
        tb = oracle.tables(**c)
        for key in ("fourT", "q", "kcorr", "kconst"):
            assert np.array_equal(tb[key], g[f"c{k}_{key}"]), (c, key)
    for k, c in enumerate(MB_TABLE_CASES):
        tb = oracle.tables(**c)
        for key in ("fourT", "q", "kcorr", "kconst"):
            assert np.array_equal(tb[key], g[f"mb{k}_{key}"]), (c, key)


@pytest.fixture(scope="module")
def pm1():
    return I.complete_pm1(2000, SEED)


def test_generator_pinned(pm1):
    g = _load("pm1_n2000.npz")
    assert _sha(pm1.dense) == str(g["J_sha256"])
    assert pm1.stats()["sumw"] == int(g["sumw"])
    k4 = I.random_kbit(800, 4, 7, pzero=1.0 / 15.0, bmax=300)
    g4 = _load("k4bias_n800.npz")
    assert _sha(k4.dense) == str(g4["J_sha256"]) and _sha(k4.bias) == str(g4["bias_sha256"])
    sp = I.random_graph(800, 4690, True, 11, bmax=2)
    gs = _load("sparse_n800.npz")
    assert _sha(sp.to_dense()) == str(gs["J_sha256"]) and _sha(sp.bias) == str(gs["bias_sha256"])


@pytest.mark.parametrize("mode", [m for m, _ in PM1_SCHEDULES])
def test_pm1_every_mode(oracle, pm1, mode):
    g = _load("pm1_n2000.npz")
    sc = dict(PM1_SCHEDULES)[mode]
    tb = oracle.tables(**sc)
    res = oracle.run_batch(2000, tb, SEED, 0, 4, dense=pm1.dense)
    sumw = int(g["sumw"])
    for trial in range(4):
        assert np.array_equal(res["spins"][trial], g[f"{mode}_{trial}_spins"])
        assert int(res["sum_sh"][trial]) == int(g[f"{mode}_{trial}_sum_sh"])
        assert int(res["flips"][trial]) == int(g[f"{mode}_{trial}_flips"])
        assert np.array_equal(res["nlin"][trial], g[f"{mode}_{trial}_nlin"])
        sh = int(res["sum_sh"][trial])
        half = sh // 2 if sh >= 0 else -((-sh) // 2)
        tot = sumw + half
        cut = tot // 2 if tot >= 0 else -((-tot) // 2)
        assert cut == int(g[f"{mode}_{trial}_cut"]) == pm1.cut(res["spins"][trial])


def test_k4_bias(oracle):
    g = _load("k4bias_n800.npz")
    k4 = I.random_kbit(800, 4, 7, pzero=1.0 / 15.0, bmax=300)
    tb = oracle.tables(S=200, t0=200.0, t1=20.0, q=40.0, lam=0.6, ramp=True)
    for trial in range(4):
        r = oracle.run(800, tb, 99, trial, dense=k4.dense, bias=k4.bias, want_h=True)
        assert np.array_equal(r["spins"], g[f"t{trial}_spins"])
        assert np.array_equal(r["nlin"], g[f"t{trial}_nlin"])
        for k in ("sum_sh", "sum_bs", "flips"):
            assert r[k] == int(g[f"t{trial}_{k}"])
        # the final fields equal a from-scratch recomputation (test_ref_bias.cpp part 2)
        assert np.array_equal(r["h"], k4.fields(r["spins"]))
        # CSR input gives the same trial
        c = oracle.run(800, tb, 99, trial, csr=k4.to_csr(), bias=k4.bias)
        assert np.array_equal(c["spins"], r["spins"]) and c["sum_sh"] == r["sum_sh"]


def test_ragged_sizes(oracle):
    g = _load("ragged_k2.npz")
    tb = oracle.tables(S=64, t0=3.0, t1=0.5, q=1.0, lam=0.5, ramp=True)
    for n in (1, 17, 257, 1000, 2048):
        inst = I.random_kbit(n, 2, 5 + n, pzero=0.3, bmax=3) if n > 1 else I.Instance(
            n=1, dense=np.zeros((1, 1), np.int8), bias=np.array([3], np.int32))
        assert _sha(inst.dense) == str(g[f"n{n}_J_sha256"])
        for trial in range(2):
            r = oracle.run(n, tb, 5, trial, dense=inst.dense, bias=inst.bias)
            assert np.array_equal(r["spins"], g[f"n{n}_t{trial}_spins"]), n
            assert np.array_equal(r["nlin"], g[f"n{n}_t{trial}_nlin"]), n
            for k in ("sum_sh", "sum_bs", "flips"):
                assert r[k] == int(g[f"n{n}_t{trial}_{k}"]), (n, k)


def test_sparse_bias(oracle):
    g = _load("sparse_n800.npz")
    sp = I.random_graph(800, 4690, True, 11, bmax=2)
    tb = oracle.tables(S=250, t0=6.0, t1=1.0, q=2.0, kappa=2.0, ramp=True)
    for trial in range(3):
        r = oracle.run(800, tb, SEED, 1000 + trial, csr=sp.to_csr(), bias=sp.bias)
        assert np.array_equal(r["spins"], g[f"t{trial}_spins"])
        assert np.array_equal(r["nlin"], g[f"t{trial}_nlin"])
        for k in ("sum_sh", "sum_bs", "flips"):
            assert r[k] == int(g[f"t{trial}_{k}"])
        assert sp.energy(r["spins"]) == -(r["sum_sh"] + r["sum_bs"]) // 2


def test_planted_mistake_is_caught(oracle, pm1):
    """A checker that cannot fail is no checker: perturb one coupling and the trace must differ."""
    g = _load("pm1_n2000.npz")
    bad = pm1.dense.copy()
    bad[3, 5] = bad[5, 3] = -bad[3, 5]
    tb = oracle.tables(**dict(PM1_SCHEDULES)["onsager"])
    r = oracle.run(2000, tb, SEED, 0, dense=bad)
    assert not np.array_equal(r["nlin"], g["onsager_0_nlin"]) or not np.array_equal(r["spins"], g["onsager_0_spins"])


def test_generalised_np(oracle):
    """n > 2048: rounds = NP / 256 with NP = ceil(n / 256) * 256; fields stay consistent with a recomputation."""
    assert oracle.lib.orc_np(2000) == 2048 and oracle.lib.orc_np(2049) == 2304 and oracle.lib.orc_np(20000) == 20224
    t = I.torus(50, 60, 3, True, bmax=2)
    tb = oracle.tables(S=100, t0=4.0, t1=0.5, q=1.0, kappa=1.5, ramp=True)
    r = oracle.run(t.n, tb, 1, 2, csr=t.to_csr(), bias=t.bias, want_h=True)
    assert np.array_equal(r["h"], t.fields(r["spins"]))
    assert r["spins"].shape == (I.spin_words(t.n),)
