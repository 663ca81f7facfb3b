"""GPU parity of the 51-instance sparse batch (uneven sizes N = 800 .. 20000: Erdos-Renyi p = 0.06 at N = 800,
degree-~6 and degree-~12 random graphs, 2-D toroidal grids; weights +1 or iid +-1; K = 2 planes with integer bias;
temperature-scaled correction) in ONE persistent launch of the plain engine (CSR path: adjacency rows in shared
memory, integer weights), against the golden-model restatement:
every spin, flip count, sum s*h, sum b*s and n_lin step of every anneal."""
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu

SCHED = dict(S=60, t0=6.0, t1=0.5, q=1.5, kappa=2.0, ramp=True)


@pytest.fixture(scope="module")
def batch(cuda):
    insts = [(name, build()) for name, build in I.sparse_classes_manifest()]
    assert len(insts) == 51 and max(i.n for _, i in insts) == 20000
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    devs = [A.DeviceInstance(i) for _, i in insts]
    for (_, i), d in zip(insts, devs):
        assert i.stats()["maxabs"] == 1 and d.info["sparse"] == 1   # K = 2 range, CSR storage
    jobs = [dict(dev=d, tb=tb, seed=20261008, trial_offset=1000 * k, nchains=2, trace=True) for k, d in enumerate(devs)]
    return insts, A.run_batch(jobs)


def test_every_instance_vs_oracle(batch, oracle):
    insts, outs = batch
    otb = oracle.tables(**SCHED)
    for k, ((name, inst), r) in enumerate(zip(insts, outs)):
        ref = oracle.run_batch(inst.n, otb, 20261008, 1000 * k, 2, csr=inst.to_csr(), bias=inst.bias)
        for c in range(2):
            assert_same(r, {kk: v[c] for kk, v in ref.items()}, c, f"{name} chain {c}")


def test_energies_rescored_on_the_host(batch):
    """Device energy E = -(sum s*h + sum b*s)/2 equals an independent rescoring of the returned spins."""
    insts, outs = batch
    for (name, inst), r in zip(insts, outs):
        e = r.energies()
        for c in range(2):
            assert int(e[c]) == inst.energy(r.spins[c]), name


def test_refused_batch_enqueues_nothing(cuda):
    """A batch that mixes a valid job with one the plain engine cannot hold (n = 60000: its fields alone need more
    shared memory than a CTA has) is refused with ANC_EINVAL before anything is enqueued: the valid job's host
    outputs keep their sentinel pattern."""
    import ctypes as C
    import numpy as np
    from anechoic_b200 import _lib
    L = _lib.load()
    small, big = I.torus(20, 40, 3, True, bmax=2), I.torus(200, 300, 4, True)
    devs = [A.DeviceInstance(small), A.DeviceInstance(big)]
    tb = A.Tables.from_schedule(A.Schedule(S=20, t0=4.0, t1=0.5, q=1.0, kappa=2.0, ramp=True))
    arr = (_lib.Job * 2)()
    keep = []
    for k, d in enumerate(devs):
        W = A.spin_words(d.n)
        bufs = dict(spins=np.full((2, W), 0x5A5A5A5A5A5A5A5A, np.uint64), sh=np.full(2, -7, np.int64),
                    bs=np.full(2, -7, np.int64), fl=np.full(2, -7, np.int64), tr=np.full((2, 20), -7, np.int32))
        keep.append(bufs)
        a = arr[k]
        a.inst, a.tb, a.seed, a.trial_offset, a.nchains = d._h.value, tb._h.value, 1, 0, 2
        a.spins, a.sum_sh, a.sum_bs = bufs["spins"].ctypes.data, bufs["sh"].ctypes.data, bufs["bs"].ctypes.data
        a.flips, a.trace = bufs["fl"].ctypes.data, bufs["tr"].ctypes.data
    o = _lib.opts("auto")
    rc = L.anc_run_batch(2, arr, C.byref(o))
    assert rc == -1 and "shared" in L.anc_last_error().decode()
    for b in keep:
        assert np.all(b["spins"] == 0x5A5A5A5A5A5A5A5A) and np.all(b["sh"] == -7) and np.all(b["tr"] == -7)
    # the valid job alone runs
    outs = A.run_batch([dict(dev=devs[0], tb=tb, seed=1, trial_offset=0, nchains=2)])
    assert int(outs[0].flips.sum()) > 0


def test_sparse_tuner_variants_agree_and_pick_is_recorded(cuda, oracle):
    """The run-time tuner of the CSR pass: every compiled variant gives the same bits (forced through the options),
    the first synchronous run records each variant's probe time and keeps the fastest for later launches."""
    import ctypes as C
    import numpy as np
    from anechoic_b200 import _lib
    L = _lib.load()
    inst = I.torus(60, 80, 11, True, bmax=2)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    v = C.c_int(7)
    us = (C.c_double * 4)()
    L.anc_sparse_tuning(dev._h, C.byref(v), us)
    assert v.value == -1                                   # not tuned before the first synchronous run
    ref = oracle.run_batch(inst.n, oracle.tables(**SCHED), 3, 40, 20, csr=inst.to_csr(), bias=inst.bias)
    outs = []
    for forced in range(1, 5):
        o = _lib.opts("plain")
        o.sparse_variant = forced
        r = A.RunResult(n=inst.n, trial_offset=40, spins=np.zeros((20, A.spin_words(inst.n)), np.uint64),
                        sum_sh=np.zeros(20, np.int64), sum_bs=np.zeros(20, np.int64), flips=np.zeros(20, np.int64),
                        trace=np.zeros((20, SCHED["S"]), np.int32))
        _lib.check(L.anc_run(dev._h, tb._h, 3, 40, 20, C.byref(o), r.spins.ctypes.data, r.sum_sh.ctypes.data,
                             r.sum_bs.ctypes.data, r.flips.ctypes.data, r.trace.ctypes.data))
        for c in range(20):
            assert_same(r, {k: val[c] for k, val in ref.items()}, c, f"variant {forced - 1} chain {c}")
        outs.append(r)
    L.anc_sparse_tuning(dev._h, C.byref(v), us)
    assert v.value == -1                                   # forced runs do not tune
    A.run(dev, tb, 3, 40, 20, engine="plain")              # the first unforced synchronous run tunes
    L.anc_sparse_tuning(dev._h, C.byref(v), us)
    assert 0 <= v.value < 4 and all(us[k] > 0 for k in range(4))
    assert us[v.value] == min(us[k] for k in range(4))


def test_csr_edge_formats_agree(cuda, oracle):
    """CSR instances with unit weights and n < 32767 keep their rows also as 16-bit edges, two per fetched word (the
    default); anc_run_opts.kernel_variant forces 32-bit (1) or 16-bit (2) edges. Both give the golden model's bits, on
    rows of odd and even length; an instance with a weight of magnitude above 1 refuses the 16-bit form."""
    import ctypes as C
    import numpy as np
    from anechoic_b200 import _lib
    L = _lib.load()
    sc = dict(S=80, t0=6.0, t1=0.5, q=1.5, kappa=2.0, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sc))
    inst = I.random_graph(3001, 9000, True, 4242, bmax=2)
    assert inst.stats()["maxabs"] == 1
    dev = A.DeviceInstance(inst)
    ref = oracle.run_batch(inst.n, oracle.tables(**sc), 5, 70, 6, csr=inst.to_csr(), bias=inst.bias)

    def run(variant):
        o = _lib.opts("plain")
        o.kernel_variant = variant
        r = A.RunResult(n=inst.n, trial_offset=70, spins=np.zeros((6, A.spin_words(inst.n)), np.uint64),
                        sum_sh=np.zeros(6, np.int64), sum_bs=np.zeros(6, np.int64), flips=np.zeros(6, np.int64),
                        trace=np.zeros((6, sc["S"]), np.int32))
        rc = L.anc_run(dev._h, tb._h, 5, 70, 6, C.byref(o), r.spins.ctypes.data, r.sum_sh.ctypes.data,
                       r.sum_bs.ctypes.data, r.flips.ctypes.data, r.trace.ctypes.data)
        return rc, r

    for variant in (0, 1, 2):
        rc, r = run(variant)
        assert rc == 0, L.anc_last_error().decode()
        for c in range(6):
            assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"edge format {variant} chain {c}")
    assert run(3)[0] == -1
    # a weight of 2: only the 32-bit form
    rp, col, val0 = (np.ascontiguousarray(a, t) for a, t in zip(inst.to_csr(), (np.int32, np.int32, np.int8)))
    # keep J symmetric: double both directions of every edge whose (min, max) pair hashes to 0 mod 7
    rows = np.repeat(np.arange(inst.n), np.diff(rp))
    lo, hi = np.minimum(rows, col), np.maximum(rows, col)
    val = np.ascontiguousarray(np.where((lo * 31 + hi) % 7 == 0, 2 * val0, val0), np.int8)
    h = C.c_void_p()
    _lib.check(L.anc_instance_create_csr(inst.n, rp.ctypes.data, col.ctypes.data, val.ctypes.data, None, C.byref(h)))
    try:
        o = _lib.opts("plain")
        o.kernel_variant = 2
        sp = np.zeros((1, A.spin_words(inst.n)), np.uint64)
        sh = np.zeros(1, np.int64)
        assert L.anc_run(h, tb._h, 5, 0, 1, C.byref(o), sp.ctypes.data, sh.ctypes.data, None, None, None) == -1
        assert "16-bit edges" in L.anc_last_error().decode()
        o.kernel_variant = 0
        _lib.check(L.anc_run(h, tb._h, 5, 0, 1, C.byref(o), sp.ctypes.data, sh.ctypes.data, None, None, None))
        ref2 = oracle.run_batch(inst.n, oracle.tables(**sc), 5, 0, 1, csr=(rp, col, val))
        assert np.array_equal(sp[0], ref2["spins"][0]) and int(sh[0]) == int(ref2["sum_sh"][0])
    finally:
        L.anc_instance_destroy(h)
