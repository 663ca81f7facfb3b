"""GPU: failure detection of the tensor engine's bounded waits, without a GPU fault.

The reference spins on its exchange barriers with no bound (gpu/onsager_v2_20261007/src/sca_gpu.cu:249). Here every
device wait of the engine's kernels has a limit (anc_set_wait_ns, default 2 s). With the limit at 0 the first wait
that is not already satisfied gives up: the kernel records an error, stops issuing work, lets the copies and MMAs it
has in flight finish (under its own fixed bound) and returns, and the call reports ANC_ETIMEOUT. The limit is then
restored and the same context and handles run the same anneals bit-exactly against the golden-model restatement.
"""
import pytest

import anechoic_b200 as A
from anechoic_b200 import _lib
from anechoic_b200 import instances as I
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu

SEED = 20261004
SCHED = dict(S=60, t0=30.0, t1=5.0, q=4.0, lam=1.05, ramp=True)


@pytest.fixture(scope="module")
def pm1(cuda):
    inst = I.complete_pm1(2000, SEED)
    return inst, A.DeviceInstance(inst)


@pytest.mark.parametrize("kind,kernel", [("fp4", "tensor-fp4"), ("int8", "tensor-int8")])
def test_forced_expiry_reports_timeout_then_runs_exactly(pm1, oracle, kind, kernel):
    inst, dev = pm1
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    L = _lib.load()
    old = L.anc_get_wait_ns()
    assert old == 2_000_000_000
    L.anc_set_wait_ns(0)
    try:
        with pytest.raises(A.AncError) as e:
            A.run(dev, tb, SEED, 0, 256, trace=True, engine="tensor", tensor_kind=kind)
        assert e.value.code == -3 and "wait" in str(e.value)
    finally:
        L.anc_set_wait_ns(old)
    assert L.anc_get_wait_ns() == old
    r = A.run(dev, tb, SEED, 0, 256, trace=True, engine="tensor", tensor_kind=kind)
    assert r.kernel == kernel
    ref = oracle.run_batch(2000, oracle.tables(**SCHED), SEED, 0, 256, dense=inst.dense)
    for c in range(256):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"{kind} after expiry, chain {c}")
