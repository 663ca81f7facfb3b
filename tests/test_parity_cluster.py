"""GPU parity of the cluster variant of the plain engine (each anneal spread over a cluster of 8 CTAs; dense 1-bit
couplings, n <= 2048) through the C ABI, against the reference's golden outputs, the golden-model restatement and the
one-CTA plain engine: every spin, every step's n_lin, flips, sum s*h, sum b*s, final fields -- bit-exact."""
import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from tests.golden.make_golden import PM1_SCHEDULES, SEED
from tests.test_parity_plain import _g, assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pm1(cuda):
    inst = I.complete_pm1(2000, SEED)
    return inst, A.DeviceInstance(inst)


@pytest.mark.parametrize("mode", [m for m, _ in PM1_SCHEDULES])
def test_golden_every_mode(pm1, mode):
    """The reference's own outputs (tests/golden/pm1_n2000.npz), trials 0..3 of each correction mode."""
    inst, dev = pm1
    g = _g("pm1_n2000.npz")
    tb = A.Tables.from_schedule(A.Schedule(**dict(PM1_SCHEDULES)[mode]))
    r = A.run(dev, tb, SEED, 0, 4, trace=True, engine="cluster")
    assert r.kernel == "plain-cluster"
    for t in range(4):
        assert np.array_equal(r.spins[t], g[f"{mode}_{t}_spins"]), (mode, t)
        assert np.array_equal(r.trace[t], g[f"{mode}_{t}_nlin"]), (mode, t)
        assert int(r.flips[t]) == int(g[f"{mode}_{t}_flips"])
        assert int(r.sum_sh[t]) == int(g[f"{mode}_{t}_sum_sh"])


def test_full_schedule_vs_oracle(pm1, oracle):
    """16 anneals, trial ids far from zero, counted Onsager over the full 1000-step default schedule, fields out."""
    inst, dev = pm1
    tb = A.Tables.from_schedule(A.Schedule(S=1000, lam=1.05, ramp=True))
    r = A.run(dev, tb, SEED, 2_000_000, 16, trace=True, fields=True, engine="cluster")
    ref = oracle.run_batch(2000, oracle.tables(S=1000, lam=1.05, ramp=True), SEED, 2_000_000, 16, dense=inst.dense)
    for c in range(16):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
        assert np.array_equal(r.fields[c], inst.fields(r.spins[c]))


def test_auto_picks_it_for_a_few_anneals(pm1):
    """AUTO runs a handful of anneals on the cluster variant, with the plain engine's results."""
    inst, dev = pm1
    tb = A.Tables.from_schedule(A.Schedule(S=300, lam=1.05, ramp=True))
    a = A.run(dev, tb, 4, 9, 4, trace=True, fields=True)
    assert a.kernel == "plain-cluster"
    b = A.run(dev, tb, 4, 9, 4, trace=True, fields=True, engine="plain")
    assert b.kernel == "plain"
    for f in ("spins", "sum_sh", "sum_bs", "flips", "trace", "fields"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


@pytest.mark.parametrize("n", [17, 257, 1000, 2047, 2048])
def test_ragged_with_bias(cuda, oracle, n):
    """Active spins fewer than the 2048 slots (padding slots still draw) and a bias."""
    inst = I.complete_pm1(n, 100 + n)
    inst.bias = np.random.default_rng(n).integers(-9, 10, n).astype(np.int32)
    dev = A.DeviceInstance(inst)
    assert dev.info["kbits"] == 1
    sc = dict(S=90, t0=12.0, t1=1.0, q=2.0, lam=0.9, ramp=True)
    r = A.run(dev, A.Tables.from_schedule(A.Schedule(**sc)), 6, 40, 3, trace=True, fields=True, engine="cluster")
    ref = oracle.run_batch(n, oracle.tables(**sc), 6, 40, 3, dense=inst.dense, bias=inst.bias)
    for c in range(3):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"n={n} chain {c}")
        assert np.array_equal(r.fields[c], inst.fields(r.spins[c]))


def test_more_anneals_than_one_wave(pm1):
    """More clusters than fit at once run in waves: 200 anneals, the same as the one-CTA plain engine."""
    inst, dev = pm1
    tb = A.Tables.from_schedule(A.Schedule(S=120, t0=15.0, q=8.0, kappa=2.0, ramp=True))
    a = A.run(dev, tb, SEED, 0, 200, trace=True, engine="cluster")
    b = A.run(dev, tb, SEED, 0, 200, trace=True, engine="plain")
    for f in ("spins", "sum_sh", "flips", "trace"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_clamped_decision(cuda, oracle):
    """A bias large enough that s*h*65536 overflows int32: the range plan's clamp, forced or automatic, is exact."""
    inst = I.complete_pm1(2000, 3)
    inst.bias = np.random.default_rng(3).integers(-30000, 30001, 2000).astype(np.int32)
    dev = A.DeviceInstance(inst)
    sc = dict(S=60, t0=400.0, t1=40.0, q=2000.0, lam=0.3, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    plan = dev.range_plan(tb)
    assert not plan["plain_ok"] and plan["hclamp"] > 0
    ref = oracle.run_batch(2000, oracle.tables(**sc), 1, 0, 2, dense=inst.dense, bias=inst.bias)
    for wide in ("auto", 1):
        r = A.run(dev, tb, 1, 0, 2, trace=True, engine="cluster", wide=wide)
        for c in range(2):
            assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"wide={wide}")


def test_refuses_other_instances(cuda):
    """Multi-bit couplings or n > 2048 are refused with ANC_EINVAL (no launch)."""
    tb = A.Tables.from_schedule(A.Schedule(S=10))
    for inst in (I.random_kbit(500, 2, 1, pzero=0.3), I.complete_pm1(2049, 1)):
        with pytest.raises(A.AncError) as e:
            A.run(A.DeviceInstance(inst), tb, 1, 0, 1, engine="cluster")
        assert e.value.code == -1 and "cluster" in str(e.value)


@pytest.mark.parametrize("variant", [1, 2])
def test_cluster_sizes_forced_vs_oracle(cuda, oracle, variant):
    """Both cluster sizes, forced through anc_run_opts.kernel_variant (1: 8 CTAs per anneal, 2: 16 CTAs, the spin and
    exchange words then interleaving two rounds' half words), with a bias, a ragged n and more anneals than one wave of
    16-CTA clusters: every spin, n_lin step, flip count and sum against the golden-model restatement."""
    import ctypes as C
    from anechoic_b200 import _lib
    L = _lib.load()
    n = 1500
    inst = I.random_kbit(n, 2, 31, pzero=0.0, bmax=5)
    dev = A.DeviceInstance(inst)
    sc = dict(S=200, t0=20.0, t1=2.0, q=4.0, lam=1.05, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    nch = 10
    ref = oracle.run_batch(n, oracle.tables(**sc), 77, 4321, nch, dense=inst.dense, bias=inst.bias)
    o = _lib.opts("cluster")
    o.kernel_variant = variant
    r = A.RunResult(n=n, trial_offset=4321, spins=np.zeros((nch, A.spin_words(n)), np.uint64),
                    sum_sh=np.zeros(nch, np.int64), sum_bs=np.zeros(nch, np.int64), flips=np.zeros(nch, np.int64),
                    trace=np.zeros((nch, sc["S"]), np.int32))
    _lib.check(L.anc_run(dev._h, tb._h, 77, 4321, nch, C.byref(o), r.spins.ctypes.data, r.sum_sh.ctypes.data,
                         r.sum_bs.ctypes.data, r.flips.ctypes.data, r.trace.ctypes.data))
    assert L.anc_last_kernel() == 4
    for c in range(nch):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"variant {variant} chain {c}")
    o.kernel_variant = 3
    assert L.anc_run(dev._h, tb._h, 77, 0, 1, C.byref(o), r.spins.ctypes.data, r.sum_sh.ctypes.data, None, None,
                     None) == -1
