"""GPU: the device-output entry points replay from a CUDA graph. anc_run_device (plain, cluster and fp4 tensor engines)
and anc_run_batch_noalloc (many uneven instances, dense and sparse, in persistent launches) are captured once into a
torch CUDA graph, after a first eager run has sized the handle's workspaces. Every replay then gives, bit for bit, the
results of eager runs of the same trial ids. The launches zero their own counters and flags as part of the captured
work, so a graph can be replayed any number of times."""
import numpy as np
import pytest
import torch

import anechoic_b200 as A
from anechoic_b200 import _lib, instances as I

pytestmark = pytest.mark.gpu

SCHED = dict(S=150, lam=1.05, ramp=True)


def _outputs(nchains, n):
    W = A.spin_words(n)
    return dict(sp=torch.zeros((nchains, W), dtype=torch.int64, device="cuda"),
                sh=torch.zeros(nchains, dtype=torch.int64, device="cuda"),
                bs=torch.zeros(nchains, dtype=torch.int64, device="cuda"),
                fl=torch.zeros(nchains, dtype=torch.int64, device="cuda"))


@pytest.mark.parametrize("engine,nchains", [("plain", 40), ("cluster", 5), ("tensor", 256)])
def test_device_runs_replay_from_a_graph(cuda, engine, nchains):
    inst = I.complete_pm1(2000, 20261004)
    dev = A.DeviceInstance(inst)
    tb = A.Tables.from_schedule(A.Schedule(**SCHED))
    L = _lib.load()
    o = _lib.opts(engine)
    outs = [_outputs(nchains, inst.n) for _ in range(2)]

    def launch(k, stream):
        b = outs[k]
        _lib.check(L.anc_run_device(dev._h, tb._h, 11, 1000 + k * nchains, nchains, o, b["sp"].data_ptr(),
                                    b["sh"].data_ptr(), b["bs"].data_ptr(), b["fl"].data_ptr(), None, stream))

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        launch(0, side.cuda_stream)            # eager: sizes the workspaces
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    kernel = _lib.last_kernel()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cs = torch.cuda.current_stream().cuda_stream
        launch(0, cs)
        launch(1, cs)
    for rep in range(2):
        for b in outs:
            for t in b.values():
                t.zero_()
        g.replay()
        torch.cuda.synchronize()
        for k in range(2):
            ref = A.run(dev, tb, 11, 1000 + k * nchains, nchains, engine=engine)
            assert ref.kernel == kernel
            b = outs[k]
            assert np.array_equal(b["sp"].cpu().numpy().view(np.uint64), ref.spins), (engine, rep, k)
            assert np.array_equal(b["sh"].cpu().numpy(), ref.sum_sh), (engine, rep, k)
            assert np.array_equal(b["fl"].cpu().numpy(), ref.flips), (engine, rep, k)


def test_uneven_batch_replays_from_a_graph(cuda):
    """anc_run_batch_noalloc: dense 1- and 4-bit and sparse instances of different sizes in one allocation-free call
    (a persistent launch per kernel kind), captured once and replayed twice; a second, different call between the
    replays does not change what the graph runs."""
    import ctypes as C
    from anechoic_b200 import noalloc
    from tests.test_zz_no_alloc import _build, _check
    sched = dict(S=90, t0=12.0, t1=1.0, q=2.0, lam=0.9, ramp=True)
    insts = [I.complete_pm1(700, 5), I.random_kbit(1300, 4, 6, pzero=0.5, bmax=5), I.torus(30, 40, 7, True, 2),
             I.random_graph(900, 4000, True, 8, 3)]
    built = [_build(inst, sched, 4, 100 * k, 6 + 5 * k, torch) for k, inst in enumerate(insts)]
    jobs = (noalloc.DeviceJob * len(built))(*[b[0] for b in built])
    L = _lib.load()

    def launch(js, stream):
        _lib.check(L.anc_run_batch_noalloc(len(js), js, C.c_void_p(stream)))

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        launch(jobs, side.cuda_stream)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        launch(jobs, torch.cuda.current_stream().cuda_stream)
    other = _build(I.complete_pm1(300, 9), sched, 5, 0, 3, torch)
    for rep in range(2):
        for _, keep, _ in built:
            for name in ("spins", "sh", "bs", "fl", "trace"):
                keep[name].zero_()
        g.replay()
        torch.cuda.synchronize()
        for k, (_, keep, ref) in enumerate(built):
            _check(keep, ref, f"job {k} replay {rep}")
        launch((noalloc.DeviceJob * 1)(other[0]), torch.cuda.current_stream().cuda_stream)   # a different call
        torch.cuda.synchronize()
        _check(other[1], other[2], "interleaved call")
