"""GPU parity of the batched tensor-core engine (tcgen05 int8 J * dS, fields in TMEM) through the C ABI against the
golden model and against the plain engine: bit-exact (integer path, no tolerance)."""
import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from tests.golden.make_golden import PM1_SCHEDULES, SEED
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pm1(cuda):
    inst = I.complete_pm1(2000, SEED)
    return inst, A.DeviceInstance(inst)


@pytest.mark.parametrize("mode", [m for m, _ in PM1_SCHEDULES])
def test_pm1_every_mode_vs_oracle(pm1, oracle, mode):
    """256 anneals (two replica groups) per correction mode; every spin, flip count and n_lin step."""
    inst, dev = pm1
    sc = dict(PM1_SCHEDULES)[mode]
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, SEED, 0, 256, trace=True, engine="tensor")
    ref = oracle.run_batch(2000, oracle.tables(**sc), SEED, 0, 256, dense=inst.dense)
    for c in range(256):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"{mode} chain {c}")


def test_golden_fixture(pm1):
    """The reference's own outputs for trials 0..3 (tests/golden/pm1_n2000.npz) via the tensor engine."""
    import os
    from tests.conftest import GOLDEN
    inst, dev = pm1
    g = np.load(os.path.join(GOLDEN, "pm1_n2000.npz"))
    for mode, sc in PM1_SCHEDULES:
        r = A.run(dev, A.Tables.from_schedule(A.Schedule(**sc)), SEED, 0, 4, trace=True, engine="tensor")
        for t in range(4):
            assert np.array_equal(r.spins[t], g[f"{mode}_{t}_spins"]), (mode, t)
            assert np.array_equal(r.trace[t], g[f"{mode}_{t}_nlin"]), (mode, t)
            assert int(r.flips[t]) == int(g[f"{mode}_{t}_flips"])


def test_ragged_chain_count_and_offset(pm1, oracle):
    """A partial replica group (130 chains) and a large trial offset; fields checked too."""
    inst, dev = pm1
    sc = dict(S=150, lam=1.05, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 7, 3_000_000, 130, trace=True, fields=True, engine="tensor")
    ref = oracle.run_batch(2000, oracle.tables(**sc), 7, 3_000_000, 130, dense=inst.dense)
    for c in range(130):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
    for c in (0, 129):
        assert np.array_equal(r.fields[c], inst.fields(r.spins[c]))


def test_tensor_equals_plain(pm1):
    """Both engines on the same 128 trials: identical results."""
    inst, dev = pm1
    tb = A.Tables.from_schedule(A.Schedule(S=300, kappa=2.0, ramp=True))
    a = A.run(dev, tb, 11, 500, 128, trace=True, engine="tensor")
    b = A.run(dev, tb, 11, 500, 128, trace=True, engine="plain")
    assert np.array_equal(a.spins, b.spins) and np.array_equal(a.trace, b.trace)
    assert np.array_equal(a.sum_sh, b.sum_sh) and np.array_equal(a.flips, b.flips)


@pytest.mark.parametrize("n,kbits,bmax", [(3000, 4, 40), (4096, 2, 0), (1000, 2, 5)])
def test_sizes_and_bias_vs_oracle(cuda, oracle, n, kbits, bmax):
    """NP = 3072 (12 rounds) with K = 4 couplings and bias, NP = 4096 (16 rounds), and n < 2048 with padding."""
    inst = I.random_kbit(n, kbits, 100 + n, pzero=0.2, bmax=bmax)
    dev = A.DeviceInstance(inst)
    sc = dict(S=60, t0=float(2 * np.sqrt(n)), t1=1.0, q=2.0, lam=0.7, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 5, 40, 130, trace=True, fields=True, engine="tensor")
    ref = oracle.run_batch(n, oracle.tables(**sc), 5, 40, 130, dense=inst.dense, bias=inst.bias)
    for c in range(130):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"n={n} chain {c}")
    assert np.array_equal(r.fields[5], inst.fields(r.spins[5]))


def test_wide_clamp_tensor(cuda, oracle):
    k2 = I.random_kbit(2000, 2, 5, pzero=0.0, bmax=30000)
    sc = dict(S=80, t0=400.0, t1=40.0, q=2000.0, lam=0.3, ramp=True)
    dev = A.DeviceInstance(k2)
    r = A.run(dev, A.Tables.from_schedule(A.Schedule(**sc)), 1, 0, 128, trace=True, engine="tensor")
    ref = oracle.run_batch(2000, oracle.tables(**sc), 1, 0, 128, dense=k2.dense, bias=k2.bias)
    for c in range(128):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
