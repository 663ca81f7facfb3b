"""GPU parity of the plain (bit-column) engine through the C ABI against the golden model: every spin, every step's
n_lin, flips, sum s*h, sum b*s -- bit-exact (integer path, no tolerance)."""
import os

import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from tests.conftest import GOLDEN
from tests.golden.make_golden import PM1_SCHEDULES, SEED

pytestmark = pytest.mark.gpu


def _g(name):
    return np.load(os.path.join(GOLDEN, name))


def assert_same(res, ref, c, ctx=""):
    """res: RunResult (chain c); ref: oracle dict for one trial."""
    assert np.array_equal(res.spins[c], ref["spins"]), f"spins differ {ctx}"
    assert int(res.sum_sh[c]) == int(ref["sum_sh"]), f"sum_sh {ctx}"
    assert int(res.sum_bs[c]) == int(ref["sum_bs"]), f"sum_bs {ctx}"
    assert int(res.flips[c]) == int(ref["flips"]), f"flips {ctx}"
    if res.trace is not None and ref.get("nlin") is not None:
        bad = np.nonzero(res.trace[c] != ref["nlin"])[0]
        assert bad.size == 0, f"n_lin differs first at step {bad[:1]} {ctx}"


@pytest.fixture(scope="module")
def pm1_dev(cuda):
    inst = I.complete_pm1(2000, SEED)
    return inst, A.DeviceInstance(inst)


@pytest.mark.parametrize("mode", [m for m, _ in PM1_SCHEDULES])
def test_pm1_golden_every_mode(pm1_dev, mode):
    """The reference's own outputs (tests/golden/pm1_n2000.npz) for trials 0..3 of each correction mode."""
    inst, dev = pm1_dev
    assert dev.info["kbits"] == 1
    g = _g("pm1_n2000.npz")
    sc = dict(PM1_SCHEDULES)[mode]
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, SEED, 0, 4, trace=True, engine="plain")
    cuts = r.cuts(dev.info["sumw"])
    for t in range(4):
        assert np.array_equal(r.spins[t], g[f"{mode}_{t}_spins"]), (mode, t)
        assert np.array_equal(r.trace[t], g[f"{mode}_{t}_nlin"]), (mode, t)
        assert int(r.flips[t]) == int(g[f"{mode}_{t}_flips"])
        assert int(r.sum_sh[t]) == int(g[f"{mode}_{t}_sum_sh"])
        assert int(cuts[t]) == int(g[f"{mode}_{t}_cut"]) == inst.cut(r.spins[t])


def test_pm1_many_chains_vs_oracle(pm1_dev, oracle):
    """64 chains, trial ids far from zero, counted Onsager at the full 1000-step default schedule."""
    inst, dev = pm1_dev
    sc = A.Schedule(S=1000, lam=1.05, ramp=True)
    tb = A.Tables.from_schedule(sc)
    r = A.run(dev, tb, SEED, 2_000_000, 64, trace=True, engine="plain")
    ref = oracle.run_batch(2000, oracle.tables(S=1000, lam=1.05, ramp=True), SEED, 2_000_000, 64, dense=inst.dense)
    for c in range(64):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")


def test_k4_bias_golden(cuda):
    g = _g("k4bias_n800.npz")
    k4 = I.random_kbit(800, 4, 7, pzero=1.0 / 15.0, bmax=300)
    dev = A.DeviceInstance(k4)
    assert dev.info["kbits"] == 4
    tb = A.Tables.from_schedule(A.Schedule(S=200, t0=200.0, t1=20.0, q=40.0, lam=0.6, ramp=True))
    r = A.run(dev, tb, 99, 0, 4, trace=True, fields=True, engine="plain")
    for t in range(4):
        ref = {k: g[f"t{t}_{k}"] for k in ("spins", "nlin", "sum_sh", "sum_bs", "flips")}
        assert_same(r, ref, t, f"trial {t}")
        assert np.array_equal(r.fields[t], k4.fields(r.spins[t]))


def test_ragged_golden(cuda):
    g = _g("ragged_k2.npz")
    tb = A.Tables.from_schedule(A.Schedule(S=64, t0=3.0, t1=0.5, q=1.0, lam=0.5, ramp=True))
    for n in (1, 17, 257, 1000, 2048):
        inst = I.random_kbit(n, 2, 5 + n, pzero=0.3, bmax=3) if n > 1 else I.Instance(
            n=1, dense=np.zeros((1, 1), np.int8), bias=np.array([3], np.int32))
        for sparse in (False, True):
            dev = A.DeviceInstance(inst, sparse=sparse)
            r = A.run(dev, tb, 5, 0, 2, trace=True, engine="plain")
            for t in range(2):
                ref = {k: g[f"n{n}_t{t}_{k}"] for k in ("spins", "nlin", "sum_sh", "sum_bs", "flips")}
                assert_same(r, ref, t, f"n={n} sparse={sparse} trial {t}")


def test_sparse_golden(cuda):
    g = _g("sparse_n800.npz")
    sp = I.random_graph(800, 4690, True, 11, bmax=2)
    tb = A.Tables.from_schedule(A.Schedule(S=250, t0=6.0, t1=1.0, q=2.0, kappa=2.0, ramp=True))
    for sparse in (True, False):
        dev = A.DeviceInstance(sp, sparse=sparse)
        r = A.run(dev, tb, SEED, 1000, 3, trace=True, engine="plain")
        for t in range(3):
            ref = {k: g[f"t{t}_{k}"] for k in ("spins", "nlin", "sum_sh", "sum_bs", "flips")}
            assert_same(r, ref, t, f"sparse={sparse} trial {t}")


@pytest.mark.parametrize("n,kbits", [(2049, 2), (3000, 4), (4096, 1)])
def test_large_dense_vs_oracle(cuda, oracle, n, kbits):
    """n > 2048 (generalised slot layout) on dense planes."""
    if kbits == 1:
        inst = I.complete_pm1(n, 77)
    else:
        inst = I.random_kbit(n, kbits, 31 + n, pzero=0.5, bmax=20)
    dev = A.DeviceInstance(inst)
    sc = dict(S=60, t0=float(np.sqrt(n)), t1=1.0, q=2.0, lam=0.8, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 3, 10, 3, trace=True, fields=True, engine="plain")
    ref = oracle.run_batch(n, oracle.tables(**sc), 3, 10, 3, dense=inst.dense, bias=inst.bias)
    for c in range(3):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"n={n} K={kbits} chain {c}")
        assert np.array_equal(r.fields[c], inst.fields(r.spins[c]))


def test_torus_20000_vs_oracle(cuda, oracle):
    """Largest config-3 shape: 2-D torus, N = 20000 (NP = 20224, 79 rounds), CSR couplings, bias."""
    t = I.torus(100, 200, 9, True, bmax=2)
    sc = dict(S=200, t0=3.0, t1=0.3, q=1.0, kappa=2.0, ramp=True)
    dev = A.DeviceInstance(t)
    r = A.run(dev, A.Tables.from_schedule(A.Schedule(**sc)), 11, 0, 4, trace=True, engine="plain")
    ref = oracle.run_batch(t.n, oracle.tables(**sc), 11, 0, 4, csr=t.to_csr(), bias=t.bias)
    for c in range(4):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"torus chain {c}")


def test_wide_clamp_is_exact(cuda, oracle):
    """Forcing the clamped decision (and the case that needs it: large fields) changes nothing."""
    k4 = I.random_kbit(2000, 2, 5, pzero=0.0, bmax=30000)   # |h| up to ~32000: s*h*65536 overflows int32
    sc = dict(S=80, t0=400.0, t1=40.0, q=2000.0, lam=0.3, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    dev = A.DeviceInstance(k4)
    plan = dev.range_plan(tb)
    assert not plan["plain_ok"] and plan["hclamp"] > 0
    ref = oracle.run_batch(2000, oracle.tables(**sc), 1, 0, 2, dense=k4.dense, bias=k4.bias)
    for wide in ("auto", 1):
        r = A.run(dev, tb, 1, 0, 2, trace=True, engine="plain", wide=wide)
        for c in range(2):
            assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"wide={wide} plan={plan}")


def test_batch_uneven_instances(cuda, oracle):
    """Several instances of different size and kind in one persistent launch (run_batch)."""
    specs = [I.random_graph(800, 19176, False, 1, bmax=2), I.torus(40, 50, 2, True, bmax=2),
             I.random_graph(1500, 4500, True, 3, bmax=2), I.random_kbit(700, 2, 4, pzero=0.4, bmax=2)]
    sc = dict(S=120, t0=5.0, t1=0.5, q=1.5, kappa=2.0, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    devs = [A.DeviceInstance(s) for s in specs]
    jobs = [dict(dev=d, tb=tb, seed=7, trial_offset=100 * k, nchains=3, trace=True) for k, d in enumerate(devs)]
    outs = A.run_batch(jobs)
    otb = oracle.tables(**sc)
    for k, (s, r) in enumerate(zip(specs, outs)):
        kw = dict(csr=s.to_csr()) if s.is_sparse else dict(dense=s.dense)
        ref = oracle.run_batch(s.n, otb, 7, 100 * k, 3, bias=s.bias, **kw)
        for c in range(3):
            assert_same(r, {kk: v[c] for kk, v in ref.items()}, c, f"job {k} chain {c}")


def test_errors_are_reported(cuda):
    """Invalid inputs return ANC_EINVAL with a message (no exception across the ABI, no CPU fallback)."""
    bad = np.zeros((4, 4), np.int8)
    bad[0, 1] = 1   # not symmetric
    with pytest.raises(A.AncError) as e:
        A.DeviceInstance(I.Instance(n=4, dense=bad))
    assert e.value.code == -1 and "symmetric" in str(e.value)
    inst = I.random_kbit(64, 4, 1, bmax=0)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(S=10, q=30000.0))   # |q| * 65536 alone overflows int32
    with pytest.raises(A.AncError) as e:
        A.run(dev, tb, 1, 0, 1, engine="plain")
    assert e.value.code == -1
