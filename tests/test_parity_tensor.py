"""GPU parity of the batched tensor-core engine (tcgen05 J * dS, fields in TMEM) through the C ABI against the golden
model and against the plain engine: bit-exact (integer path, no tolerance). Both operand formats run on the N=2000 +-1
instance: int8 (kind::i8, int32 accumulation) and packed e2m1 (kind::mxf4, unit block scales, fp32 accumulation)."""
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


KINDS = ("int8", "fp4")
_ORACLE_CACHE = {}


def _oracle_pm1(oracle, inst, mode, sc):
    if mode not in _ORACLE_CACHE:
        _ORACLE_CACHE[mode] = oracle.run_batch(2000, oracle.tables(**sc), SEED, 0, 256, dense=inst.dense)
    return _ORACLE_CACHE[mode]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("mode", [m for m, _ in PM1_SCHEDULES])
def test_pm1_every_mode_vs_oracle(pm1, oracle, mode, kind):
    """256 anneals (two replica groups) per correction mode; every spin, flip count and n_lin step."""
    inst, dev = pm1
    sc = dict(PM1_SCHEDULES)[mode]
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, SEED, 0, 256, trace=True, engine="tensor", tensor_kind=kind)
    assert r.kernel == f"tensor-{kind}"
    ref = _oracle_pm1(oracle, inst, mode, sc)
    for c in range(256):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"{mode} {kind} chain {c}")


@pytest.mark.parametrize("kind", KINDS)
def test_golden_fixture(pm1, kind):
    """The reference's own outputs for trials 0..3 (tests/golden/pm1_n2000.npz) via the tensor engine."""
    import os
    from tests.conftest import GOLDEN
    inst, dev = pm1
    g = np.load(os.path.join(GOLDEN, "pm1_n2000.npz"))
    for mode, sc in PM1_SCHEDULES:
        r = A.run(dev, A.Tables.from_schedule(A.Schedule(**sc)), SEED, 0, 4, trace=True, engine="tensor",
                  tensor_kind=kind)
        for t in range(4):
            assert np.array_equal(r.spins[t], g[f"{mode}_{t}_spins"]), (mode, t)
            assert np.array_equal(r.trace[t], g[f"{mode}_{t}_nlin"]), (mode, t)
            assert int(r.flips[t]) == int(g[f"{mode}_{t}_flips"])


@pytest.mark.parametrize("kind", KINDS)
def test_ragged_chain_count_and_offset(pm1, oracle, kind):
    """A partial replica group (130 chains) and a large trial offset; fields checked too."""
    inst, dev = pm1
    sc = dict(S=150, lam=1.05, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 7, 3_000_000, 130, trace=True, fields=True, engine="tensor", tensor_kind=kind)
    ref = oracle.run_batch(2000, oracle.tables(**sc), 7, 3_000_000, 130, dense=inst.dense)
    for c in range(130):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
    for c in (0, 129):
        assert np.array_equal(r.fields[c], inst.fields(r.spins[c]))


@pytest.mark.parametrize("kind", KINDS)
def test_tensor_equals_plain(pm1, kind):
    """Both engines on the same 1100 trials: more replica groups than co-resident slots, so CTAs run a second round
    (its fields must be set before tiles from faster slices are accumulated). Identical results."""
    inst, dev = pm1
    tb = A.Tables.from_schedule(A.Schedule(S=300, kappa=2.0, ramp=True))
    a = A.run(dev, tb, 11, 500, 1100, trace=True, engine="tensor", tensor_kind=kind)
    b = A.run(dev, tb, 11, 500, 1100, trace=True, engine="plain")
    assert np.array_equal(a.spins, b.spins) and np.array_equal(a.trace, b.trace)
    assert np.array_equal(a.sum_sh, b.sum_sh) and np.array_equal(a.flips, b.flips)


def test_fp4_with_large_bias_vs_oracle(cuda, oracle):
    """K=2 couplings (|J| <= 1) with bias up to 6000: fields reach ~7600, inside the fp4 kernel's exact range."""
    inst = I.random_kbit(2000, 2, 91, pzero=0.2, bmax=6000)
    dev = A.DeviceInstance(inst)
    sc = dict(S=120, t0=3000.0, t1=50.0, q=4.0, lam=0.7, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 3, 9, 200, trace=True, fields=True, engine="tensor", tensor_kind="fp4")
    assert r.kernel == "tensor-fp4"
    ref = oracle.run_batch(2000, oracle.tables(**sc), 3, 9, 200, dense=inst.dense, bias=inst.bias)
    for c in range(200):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
    for c in (0, 199):
        assert np.array_equal(r.fields[c], inst.fields(r.spins[c]))


def test_fp4_refuses_wide_couplings(cuda):
    """Forcing the fp4 format on K=4 couplings is an argument error (no launch)."""
    inst = I.random_kbit(2000, 4, 5, pzero=0.2)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(S=10, t0=60.0, t1=2.0, q=2.0, lam=0.7))
    with pytest.raises(A.AncError) as e:
        A.run(dev, tb, 1, 0, 128, engine="tensor", tensor_kind="fp4")
    assert e.value.code == -1
    r = A.run(dev, tb, 1, 0, 128, engine="tensor")
    assert r.kernel == "tensor-int8"


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
