"""GPU parity of the plain engine's streaming layout (the N = 16384 dense stress instances of uneven coupling width:
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
