"""GPU: schedules longer than the reference runner's limit (sca_gpu.cu: S <= 4096; the tg variant reads tables from
global memory up to 65536): the engines read every table from global memory, so S = 20000 runs bit-exact on both."""
import pytest

import anechoic_b200 as A
from anechoic_b200 import instances as I
from tests.test_parity_plain import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("engine", ["plain", "tensor"])
def test_s20000_vs_oracle(cuda, oracle, engine):
    inst = I.random_kbit(300, 2, 31, pzero=0.3, bmax=2)
    sc = dict(S=20000, t0=20.0, t1=0.2, q=1.0, lam=1.05, ramp=True)
    r = A.run(A.DeviceInstance(inst), A.Tables.from_schedule(A.Schedule(**sc)), 4, 0, 4, trace=True, engine=engine)
    ref = oracle.run_batch(300, oracle.tables(**sc), 4, 0, 4, dense=inst.dense, bias=inst.bias)
    for c in range(4):
        assert_same(r, {k: v[c] for k, v in ref.items()}, c, f"{engine} chain {c}")
