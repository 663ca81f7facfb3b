"""GPU: the run-time tuner of the dense kernels' compiled variants (anc_kernel_tuning) -- the plain engine's rows per
batch on dense instances (K = 1: three variants, K = 2: two) and the fp4 kernel's ring depth (4, 6, 5 or 3 stages).
Every variant, forced through anc_run_opts.kernel_variant, gives the golden model's bits; after a synchronous run the
run's tuning key holds a probe time for every variant and the tuner's choice from them; variants out of range are refused
before anything is launched."""
import ctypes as C

import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import _lib
from anechoic_b200 import instances as I
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu

SCHED = dict(S=120, t0=20.0, t1=2.0, q=4.0, lam=1.05, ramp=True)
KERNEL_PLAIN, KERNEL_FP4 = 1, 3


def _run(L, dev, tb, seed, off, nchains, o, S):
    r = A.RunResult(n=dev.n, trial_offset=off, spins=np.zeros((nchains, A.spin_words(dev.n)), np.uint64),
                    sum_sh=np.zeros(nchains, np.int64), sum_bs=np.zeros(nchains, np.int64),
                    flips=np.zeros(nchains, np.int64), trace=np.zeros((nchains, S), np.int32))
    _lib.check(L.anc_run(dev._h, tb._h, seed, off, nchains, C.byref(o), r.spins.ctypes.data, r.sum_sh.ctypes.data,
                         r.sum_bs.ctypes.data, r.flips.ctypes.data, r.trace.ctypes.data))
    return r


def _rule(us):
    """The tuner's choice from its probe times: variant 0 unless another is more than 1 % faster, then the fastest."""
    best = min(range(len(us)), key=lambda k: us[k])
    return best if us[best] < 0.99 * us[0] else 0


def _tuning(L, dev, kernel, nchains):
    v, nv = C.c_int(-7), C.c_int(0)
    us = (C.c_double * 4)()
    _lib.check(L.anc_kernel_tuning(dev._h, kernel, nchains, C.byref(v), C.byref(nv), us))
    return v.value, nv.value, [us[k] for k in range(nv.value)]


@pytest.mark.parametrize("case", ["k1_n700", "k2_n1000"])
def test_plain_dense_variants_agree_and_tune(cuda, oracle, case):
    L = _lib.load()
    inst = I.complete_pm1(700, 5) if case == "k1_n700" else I.random_kbit(1000, 2, 6, pzero=0.5, bmax=3)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    ref = oracle.run_batch(inst.n, oracle.tables(**SCHED), 9, 300, 12, dense=inst.dense, bias=inst.bias)
    _, nv, _ = _tuning(L, dev, KERNEL_PLAIN, 12)
    assert nv == (3 if case == "k1_n700" else 2)
    for forced in range(1, nv + 1):
        o = _lib.opts("plain")
        o.kernel_variant = forced
        r = _run(L, dev, tb, 9, 300, 12, o, SCHED["S"])
        for c in range(12):
            assert_same(r, {k: val[c] for k, val in ref.items()}, c, f"{case} variant {forced - 1} chain {c}")
    o = _lib.opts("plain")
    o.kernel_variant = nv + 1
    spins = np.full((2, A.spin_words(inst.n)), 0x5A5A5A5A5A5A5A5A, np.uint64)
    sh = np.full(2, -7, np.int64)
    rc = L.anc_run(dev._h, tb._h, 9, 0, 2, C.byref(o), spins.ctypes.data, sh.ctypes.data, None, None, None)
    assert rc == -1 and "kernel_variant" in L.anc_last_error().decode()
    assert np.all(spins == 0x5A5A5A5A5A5A5A5A) and np.all(sh == -7)
    A.run(dev, tb, 9, 300, 12, engine="plain")              # a synchronous run tunes the key if it was not yet
    v, nv, us = _tuning(L, dev, KERNEL_PLAIN, 12)
    assert 0 <= v < nv and all(us[k] > 0 for k in range(nv))
    assert _rule(us) == v
    r = A.run(dev, tb, 9, 300, 12, engine="plain", trace=True)     # the tuned variant: same bits
    for c in range(12):
        assert_same(r, {k: val[c] for k, val in ref.items()}, c, f"{case} tuned variant {v} chain {c}")


def test_fp4_ring_depths_agree_and_tune(cuda, oracle):
    L = _lib.load()
    inst = I.complete_pm1(2000, 20261004)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    nchains = 130                                             # a full replica group and a partial one
    ref = oracle.run_batch(inst.n, oracle.tables(**SCHED), 17, 5000, nchains, dense=inst.dense)
    for forced in range(1, 5):
        o = _lib.opts("tensor", tensor_kind="fp4")
        o.kernel_variant = forced
        r = _run(L, dev, tb, 17, 5000, nchains, o, SCHED["S"])
        assert L.anc_last_kernel() == KERNEL_FP4
        for c in range(nchains):
            assert_same(r, {k: val[c] for k, val in ref.items()}, c, f"stages variant {forced - 1} chain {c}")
    o = _lib.opts("tensor", tensor_kind="fp4")
    o.kernel_variant = 5
    spins = np.zeros((2, A.spin_words(inst.n)), np.uint64)
    sh = np.zeros(2, np.int64)
    rc = L.anc_run(dev._h, tb._h, 17, 0, 2, C.byref(o), spins.ctypes.data, sh.ctypes.data, None, None, None)
    assert rc == -1 and "kernel_variant" in L.anc_last_error().decode()
    A.run(dev, tb, 17, 5000, nchains, engine="tensor")
    v, nv, us = _tuning(L, dev, KERNEL_FP4, nchains)
    assert nv == 4 and 0 <= v < 4 and all(x > 0 for x in us) and _rule(us) == v
    with pytest.raises(A.AncError):
        _tuning(L, dev, 2, nchains)                           # the int8 kernel has no variants to tune
