"""GPU: the allocation-free entry point anc_run_batch_noalloc gives the same results as anc_run, on two calls in a row.

It serves callers that cannot call cudaMalloc (their device memory is owned by their own pool or allocator, or held
to a fixed budget): every input and output below lives in memory the caller allocated beforehand (here: torch
tensors), and the library only uses its fixed scratch array. The comparison is bit-exact, as for every engine test.
This file is collected last so that a run stopping at the first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

import anechoic_b200 as A
from anechoic_b200 import noalloc

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _build(inst, sched, seed, off, nchains, torch, with_ref=True):
    """Caller-owned device inputs and outputs for one job, plus the same job through anc_run for comparison."""
    kbits = 0 if inst.is_sparse else inst.kbits()
    tb = noalloc.schedule_tables(**sched)
    keep = {"tb": {k: _dev(v, torch) for k, v in tb.items()}}
    j = noalloc.DeviceJob()
    j.n, j.kbits, j.S = inst.n, kbits, len(tb["fourT"])
    if kbits:
        keep["planes"] = _dev(noalloc.pack_planes(inst.dense, kbits).view(np.int32), torch)
        j.planes = keep["planes"].data_ptr()
    else:
        rp, adj = noalloc.pack_csr(inst)
        keep["rp"], keep["adj"] = _dev(rp, torch), _dev(adj.view(np.int32), torch)
        j.row_ptr, j.adj = keep["rp"].data_ptr(), keep["adj"].data_ptr()
    if inst.bias is not None:
        keep["bias"] = _dev(inst.bias, torch)
        j.bias = keep["bias"].data_ptr()
    for name in ("fourT", "q", "kcorr", "kconst"):
        setattr(j, name, keep["tb"][name].data_ptr())
    j.hclamp = noalloc.clamp_for(inst, tb)
    j.seed, j.trial_offset, j.nchains = seed, off, nchains
    W = A.spin_words(inst.n)
    keep["spins"] = torch.zeros((nchains, W), dtype=torch.int64, device="cuda")
    keep["sh"], keep["bs"], keep["fl"] = (torch.zeros(nchains, dtype=torch.int64, device="cuda") for _ in range(3))
    keep["trace"] = torch.zeros((nchains, j.S), dtype=torch.int32, device="cuda")
    j.spins, j.sum_sh, j.sum_bs = keep["spins"].data_ptr(), keep["sh"].data_ptr(), keep["bs"].data_ptr()
    j.flips, j.trace = keep["fl"].data_ptr(), keep["trace"].data_ptr()
    if not with_ref:
        return j, keep, None
    ref = A.run(A.DeviceInstance(inst), A.Tables.from_schedule(A.Schedule(**sched)), seed, off, nchains, trace=True,
                engine="plain")
    return j, keep, ref


def _check(keep, ref, what):
    assert np.array_equal(keep["spins"].cpu().numpy().view(np.uint64), ref.spins), what
    assert np.array_equal(keep["sh"].cpu().numpy(), ref.sum_sh), what
    assert np.array_equal(keep["bs"].cpu().numpy(), ref.sum_bs), what
    assert np.array_equal(keep["fl"].cpu().numpy(), ref.flips), what
    assert np.array_equal(keep["trace"].cpu().numpy(), ref.trace), what


def test_noalloc_matches_anc_run_twice(cuda):
    import torch
    cases = [
        (A.complete_pm1(2000, 20261004), dict(S=200, lam=1.05, ramp=True), 20261004, 0, 24),
        (A.random_kbit(1500, 4, 17, pzero=0.3, bmax=40), dict(S=120, t0=60.0, t1=2.0, q=3.0, kappa=2.0, ramp=True), 9, 50, 16),
        (A.torus(40, 60, 3, True, bmax=2), dict(S=150, t0=4.0, t1=0.5, q=1.0, kappa=2.0, ramp=True), 5, 7, 12),
    ]
    built = [_build(inst, sc, seed, off, nch, torch) for inst, sc, seed, off, nch in cases]
    jobs = (noalloc.DeviceJob * len(built))(*[b[0] for b in built])
    stream = torch.cuda.current_stream()
    for call in range(2):
        for _, keep, _ in built:
            for k in ("spins", "sh", "bs", "fl", "trace"):
                keep[k].zero_()
        noalloc.run_batch_noalloc(jobs, stream.cuda_stream)
        torch.cuda.synchronize()
        for k, (_, keep, ref) in enumerate(built):
            _check(keep, ref, f"call {call} job {k}")


def test_noalloc_rejects_oversized_requests(cuda):
    """More anneals or jobs than the fixed scratch holds: ANC_EINVAL, nothing launched. The job's buffers are real and
    sized for the whole request, so even a launch would stay in bounds."""
    import torch
    inst = A.torus(10, 10, 1, True)
    j, keep, _ = _build(inst, dict(S=2, t0=2.0, t1=1.0, q=1.0), 1, 0, 16385, torch)
    with pytest.raises(A.AncError) as e:
        noalloc.run_batch_noalloc([j])
    assert e.value.code == -1 and "16384" in str(e.value)
    with pytest.raises(A.AncError) as e:
        noalloc.run_batch_noalloc([j for _ in range(65)])
    assert e.value.code == -1 and "jobs" in str(e.value)


def test_noalloc_refused_call_enqueues_nothing(cuda):
    """A call that mixes a valid job with one the plain engine cannot hold (n = 60000: its fields alone need more
    shared memory than a CTA has) returns ANC_EINVAL before it enqueues anything: the valid job's device outputs keep
    their sentinel pattern. Both jobs' buffers are real and sized for their jobs."""
    import torch
    good = _build(A.torus(20, 40, 3, True, bmax=2), dict(S=20, t0=4.0, t1=0.5, q=1.0, kappa=2.0, ramp=True), 1, 0, 4,
                  torch)
    bad = _build(A.torus(200, 300, 4, True), dict(S=2, t0=4.0, t1=0.5, q=1.0), 1, 0, 1, torch, with_ref=False)
    for k in ("spins", "sh", "bs", "fl", "trace"):
        good[1][k].fill_(-7)
    stream = torch.cuda.current_stream()
    with pytest.raises(A.AncError) as e:
        noalloc.run_batch_noalloc([good[0], bad[0]], stream.cuda_stream)
    assert e.value.code == -1 and "shared" in str(e.value)
    torch.cuda.synchronize()
    for k in ("spins", "sh", "bs", "fl", "trace"):
        assert bool((good[1][k] == -7).all()), k
