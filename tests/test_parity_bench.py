"""GPU parity at exactly the configurations bench.py times, through the C ABI, bit-exact (integer path, no tolerance):

- the headline batch: N = 2000 +-1 instance (seed 20261004), 1024 anneals x S = 1000, counted Onsager lambda 1.05
  with ramp, t0 30, t1 5, q 4, on the packed-e2m1 tensor kernel and on AUTO, with the trial ids of bench.py's last
  timed batch of a 20-step run (trial_base + 19 * 1024 + c); every spin, flip count, sum s*h and per-step n_lin
  against the multithreaded golden-model restatement;
- config 3 at the bench schedule: the 51 sparse instances in one persistent launch at S = 1000, 4 anneals each,
  against the restatement;
- config 5 at the bench size: N = 16384, K = 4 couplings with bias, all 256 anneals at S = 5000 on the streaming
  tensor kernel against the plain engine, with the range plan's clamp active.
"""
import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from anechoic_b200 import replicas
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu

HEADLINE = dict(S=1000, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True)
SEED = 20261004
CHAINS = 1024


@pytest.fixture(scope="module")
def headline(cuda, oracle):
    inst = I.complete_pm1(2000, SEED)
    dev = A.DeviceInstance(inst)
    off = replicas.trial_base(0) + 19 * CHAINS
    ref = oracle.run_batch(2000, oracle.tables(**HEADLINE), SEED, off, CHAINS, dense=inst.dense, trace=True)
    return inst, dev, off, ref


@pytest.mark.parametrize("engine,kind", [("tensor", "fp4"), ("auto", "auto")])
def test_headline_batch_vs_oracle(headline, engine, kind):
    inst, dev, off, ref = headline
    tb = A.Tables.from_schedule(A.Schedule(**HEADLINE))
    r = A.run(dev, tb, SEED, off, CHAINS, trace=True, engine=engine, tensor_kind=kind)
    if engine == "tensor":
        assert r.kernel == "tensor-fp4"
    for c in range(CHAINS):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"{engine} chain {c}")


def test_headline_batch_device_path_matches(headline):
    """The bench's timed call (anc_run_device: device outputs, no trace) returns the same spins, sums and flips."""
    import torch
    from anechoic_b200 import _lib
    inst, dev, off, ref = headline
    tb = A.Tables.from_schedule(A.Schedule(**HEADLINE))
    W = A.spin_words(2000)
    sp = torch.zeros((CHAINS, W), dtype=torch.int64, device="cuda")
    sh, bs, fl = (torch.zeros(CHAINS, dtype=torch.int64, device="cuda") for _ in range(3))
    L = _lib.load()
    o = _lib.opts("auto")
    _lib.check(L.anc_run_device(dev._h, tb._h, SEED, off, CHAINS, o, sp.data_ptr(), sh.data_ptr(), bs.data_ptr(),
                                fl.data_ptr(), None, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert np.array_equal(sp.cpu().numpy().view(np.uint64), ref["spins"])
    assert np.array_equal(sh.cpu().numpy(), ref["sum_sh"]) and np.array_equal(fl.cpu().numpy(), ref["flips"])


def test_sparse51_at_bench_schedule_vs_oracle(cuda, oracle):
    sched = dict(S=1000, t0=6.0, t1=0.5, q=1.5, kappa=2.0, ramp=True)
    insts = [(name, build()) for name, build in I.sparse_classes_manifest()]
    tb = A.Tables.from_schedule(A.Schedule(**sched))
    devs = [A.DeviceInstance(i) for _, i in insts]
    jobs = [dict(dev=d, tb=tb, seed=SEED, trial_offset=(3 << 12) + 64 * k, nchains=4, trace=True)
            for k, d in enumerate(devs)]
    outs = A.run_batch(jobs)
    otb = oracle.tables(**sched)
    for k, ((name, inst), r) in enumerate(zip(insts, outs)):
        ref = oracle.run_batch(inst.n, otb, SEED, (3 << 12) + 64 * k, 4, csr=inst.to_csr(), bias=inst.bias)
        for c in range(4):
            assert_same(r, {kk: v[c] for kk, v in ref.items()}, c, f"{name} chain {c}")


def test_dense16k_stream_equals_plain_at_bench_size(cuda):
    inst = I.random_kbit(16384, 4, 20261009, pzero=0.0, bmax=7)
    dev = A.DeviceInstance(inst)
    sched = dict(S=5000, t0=float(2 * np.sqrt(16384) * 4), t1=2.0, q=4.0, lam=1.05, ramp=True)
    tb = A.Tables.from_schedule(A.Schedule(**sched))
    plan = dev.range_plan(tb)
    assert not plan["plain_ok"] and plan["hclamp"] > 0          # the exact clamp is active at this size
    a = A.run(dev, tb, SEED, 0, 256, trace=True, engine="tensor")
    assert a.kernel == "tensor-int8"
    b = A.run(dev, tb, SEED, 0, 256, trace=True, engine="plain")
    assert np.array_equal(a.spins, b.spins) and np.array_equal(a.trace, b.trace)
    assert np.array_equal(a.sum_sh, b.sum_sh) and np.array_equal(a.sum_bs, b.sum_bs)
    assert np.array_equal(a.flips, b.flips)
