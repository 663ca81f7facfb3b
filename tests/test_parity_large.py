"""GPU parity at large N: the tensor engine's streaming kernel (J streamed from HBM each step, NP in (8192, 16384])
and the plain engine's streaming layout (the N = 16384 dense stress instances of uneven coupling width:
the per-set counters of K = 2 / 4 planes exceed shared memory there, so each sign/magnitude set is added into the
fields as soon as it is complete) against the golden-model restatement: every spin, flip count, sum s*h, sum b*s
and n_lin step."""
import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("K,bmax", [(4, 7), (2, 3)])
def test_n16384_vs_oracle(cuda, oracle, K, bmax):
    inst = I.random_kbit(16384, K, 20261009 + K, pzero=0.0 if K == 4 else 0.2, bmax=bmax)
    dev = A.DeviceInstance(inst)
    assert dev.info["kbits"] == K and dev.info["np"] == 16384
    sc = dict(S=12, t0=float(2 * np.sqrt(16384) * (1 << (K - 1))), t1=2.0, q=4.0, lam=1.05, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 5, 77, 2, trace=True, fields=True, engine="plain")
    ref = oracle.run_batch(16384, oracle.tables(**sc), 5, 77, 2, dense=inst.dense, bias=inst.bias)
    for c in range(2):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"K={K} chain {c}")
    assert np.array_equal(r.fields[1], inst.fields(r.spins[1]))


@pytest.fixture(scope="module")
def k4_16384(cuda):
    inst = I.random_kbit(16384, 4, 20261013, pzero=0.0, bmax=7)
    return inst, A.DeviceInstance(inst)


K4_SCHED = dict(S=10, t0=1024.0, t1=2.0, q=4.0, lam=1.05, ramp=True)


def test_stream_kernel_vs_oracle(k4_16384, oracle):
    """Config 5's instance (N = 16384, K = 4, bias): 130 anneals (a full and a partial replica group)."""
    inst, dev = k4_16384
    tb = A.Tables.from_schedule(A.Schedule(**K4_SCHED))
    r = A.run(dev, tb, 3, 500, 130, trace=True, fields=True, engine="tensor")
    assert r.kernel == "tensor-int8"
    ref = oracle.run_batch(16384, oracle.tables(**K4_SCHED), 3, 500, 130, dense=inst.dense, bias=inst.bias)
    for c in range(130):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
    assert np.array_equal(r.fields[129], inst.fields(r.spins[129]))


def test_stream_kernel_equals_plain(k4_16384):
    """300 anneals: two rounds of replica-group pairs on the same CTAs (the second pair's fields must be set before
    the first tiles of other slices are accumulated)."""
    inst, dev = k4_16384
    sc = dict(K4_SCHED, S=25)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    a = A.run(dev, tb, 8, 0, 300, trace=True, engine="tensor")
    b = A.run(dev, tb, 8, 0, 300, trace=True, engine="plain")
    assert np.array_equal(a.spins, b.spins) and np.array_equal(a.trace, b.trace)
    assert np.array_equal(a.sum_sh, b.sum_sh) and np.array_equal(a.sum_bs, b.sum_bs)
    assert np.array_equal(a.flips, b.flips)


def test_stream_kernel_padded_rounds(cuda, oracle):
    """n = 9000: NP = 9216, 36 rounds, so 28 of each lane's 64 columns are padding."""
    inst = I.random_kbit(9000, 2, 77, pzero=0.3, bmax=2)
    dev = A.DeviceInstance(inst)
    sc = dict(S=15, t0=80.0, t1=1.0, q=2.0, kappa=2.0, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    r = A.run(dev, tb, 2, 9, 40, trace=True, engine="tensor")
    ref = oracle.run_batch(9000, oracle.tables(**sc), 2, 9, 40, dense=inst.dense, bias=inst.bias)
    for c in range(40):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"chain {c}")
