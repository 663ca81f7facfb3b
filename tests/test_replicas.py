"""Multi-rank replica scaling on CPU (gloo, world size 2): disjoint trial-id ranges per rank, max-over-ranks timing,
summed success counts; and the union of the ranks' anneals equals one rank running every trial (the golden-model
restatement checks it, since an anneal is a pure function of its trial id)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from anechoic_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    from anechoic_b200 import instances as I
    from oracle.oracle import Restatement
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        t = replicas.reduce_max(1.5 + rank)
        sums = replicas.reduce_sum([rank + 1, 10 * rank, 7])
        inst = I.random_kbit(96, 2, 3, pzero=0.2, bmax=2)
        orc = Restatement()
        tb = orc.tables(S=30, t0=8.0, t1=0.5, q=1.0, lam=1.05, ramp=True)
        base = replicas.trial_base(rank)
        r = orc.run_batch(96, tb, 9, base, 3, dense=inst.dense, bias=inst.bias, threads=1)
        q.put((rank, t, sums, base, r["spins"], r["flips"]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(o[1] == 2.5 for o in out)                      # max over ranks
    assert all(o[2] == [3, 10, 14] for o in out)              # sums over ranks
    bases = [o[3] for o in out]
    assert bases == [0, replicas.TRIALS_PER_RANK]             # disjoint trial-id ranges
    # one process running both ranges gives the same anneals
    from anechoic_b200 import instances as I
    from oracle.oracle import Restatement
    inst = I.random_kbit(96, 2, 3, pzero=0.2, bmax=2)
    orc = Restatement()
    tb = orc.tables(S=30, t0=8.0, t1=0.5, q=1.0, lam=1.05, ramp=True)
    for rank, _, _, base, spins, flips in out:
        ref = orc.run_batch(96, tb, 9, base, 3, dense=inst.dense, bias=inst.bias)
        assert np.array_equal(spins, ref["spins"]) and np.array_equal(flips, ref["flips"])


def test_single_process_identity():
    assert replicas.reduce_max(3.0) == 3.0 and replicas.reduce_sum([1, 2]) == [1, 2]
