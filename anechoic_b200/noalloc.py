"""Allocation-free use of the plain engine (``anc_run_batch_noalloc``): helpers for callers that own all device memory.

Some callers cannot call cudaMalloc -- an application whose device memory is entirely owned by its own pool or caching
allocator, or one held to a fixed device-memory budget. They pack the couplings themselves into the layout below,
place inputs and outputs in memory they already own, and call ``run_batch_noalloc``; the library allocates nothing and
uses one fixed scratch array (at most 64 jobs and 16384 anneals per call).

Layouts (as include/anechoic.h documents):
* dense, kbits 1/2/4: ``[kbits][NP][NWJ]`` uint32 with NP = max(2048, ceil(n/256)*256), NWJ = ceil(NP/32) rounded up
  to a multiple of 32; bit y%32 of word x*NWJ + y/32 of plane p: kbits 1 -> [J_xy = +1]; kbits 2/4 -> plane 0 =
  [J_xy < 0], plane b = bit b-1 of |J_xy|.
* CSR (kbits 0): row_ptr[n+1] int32 and adj[k] = (y << 8) | uint8(J_xy) uint32 for every nonzero of row x.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .instances import Instance, pad_spins


class DeviceJob(C.Structure):
    """ctypes mirror of anc_device_job (every pointer is device memory)."""
    _fields_ = [("n", C.c_int), ("kbits", C.c_int), ("planes", C.c_void_p), ("row_ptr", C.c_void_p),
                ("adj", C.c_void_p), ("bias", C.c_void_p), ("fourT", C.c_void_p), ("q", C.c_void_p),
                ("kcorr", C.c_void_p), ("kconst", C.c_void_p), ("S", C.c_int), ("hclamp", C.c_int32),
                ("seed", C.c_uint64), ("trial_offset", C.c_uint32), ("nchains", C.c_int), ("spins", C.c_void_p),
                ("sum_sh", C.c_void_p), ("sum_bs", C.c_void_p), ("flips", C.c_void_p), ("trace", C.c_void_p)]


def pack_planes(J: np.ndarray, kbits: int) -> np.ndarray:
    """Dense couplings (n x n int8) -> the plane words ([kbits][NP][NWJ] uint32)."""
    J = np.asarray(J, np.int8)
    n = J.shape[0]
    NP = pad_spins(n)
    NWJ = -(-(NP // 32) // 32) * 32
    if kbits == 1:
        bits = [(J == 1)]
    elif kbits in (2, 4):
        a = np.abs(J.astype(np.int16))
        bits = [(J < 0)] + [((a >> (b - 1)) & 1).astype(bool) for b in range(1, kbits)]
    else:
        raise ValueError("kbits must be 1, 2 or 4")
    out = np.zeros((kbits, NP, NWJ), np.uint32)
    for p, bm in enumerate(bits):
        padded = np.zeros((n, NWJ * 32), np.uint8)
        padded[:, :n] = bm
        words = np.packbits(padded, axis=1, bitorder="little").view("<u4")
        out[p, :n, :] = words
    return out


def pack_csr(inst: Instance):
    """CSR rows -> (row_ptr int32 [n+1], adj uint32 [nnz])."""
    rp, col, val = inst.to_csr()
    adj = (col.astype(np.uint32) << np.uint32(8)) | val.view(np.uint8).astype(np.uint32)
    return np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(adj, np.uint32)


def schedule_tables(S, t0=30.0, t1=5.0, q=4.0, lam=0.0, jv=0.0, kappa=0.0, ramp=False, scale=1.0) -> dict:
    """Host-side fixed-point tables (anc_schedule_tables; no device allocation)."""
    L = _lib.load()
    f = np.zeros(S, np.int32); qq = np.zeros(S, np.int32); kc = np.zeros(S, np.int64); ks = np.zeros(S, np.int32)
    _lib.check(L.anc_schedule_tables(S, t0, t1, q, lam, jv, kappa, int(bool(ramp)), scale, f.ctypes.data,
                                     qq.ctypes.data, kc.ctypes.data, ks.ctypes.data))
    return dict(fourT=f, q=qq, kcorr=kc, kconst=ks)


def clamp_for(inst: Instance, tb: dict) -> int:
    """hclamp for a job: 0 when the unclamped int32 decision is proven safe, else the plan's clamp."""
    L = _lib.load()
    st = inst.stats()
    ok = C.c_int(); hc = C.c_int32()
    _lib.check(L.anc_plan_ranges(inst.n, st["hmax"], st["bmax"], tb["fourT"].ctypes.data, tb["q"].ctypes.data,
                                 tb["kcorr"].ctypes.data, tb["kconst"].ctypes.data, len(tb["fourT"]), C.byref(ok),
                                 C.byref(hc)))
    return 0 if ok.value else int(hc.value)


def run_batch_noalloc(jobs, stream: int = 0):
    """Launch a list of DeviceJob (or one ctypes array) through anc_run_batch_noalloc on `stream` (a cudaStream_t
    handle as an int, 0 = default). Asynchronous: synchronise the stream before reading the outputs."""
    L = _lib.load()
    if not hasattr(L, "_noalloc_ready"):
        L.anc_run_batch_noalloc.argtypes = [C.c_int, C.POINTER(DeviceJob), C.c_void_p]
        L._noalloc_ready = True
    arr = jobs if isinstance(jobs, C.Array) else (DeviceJob * len(jobs))(*jobs)
    _lib.check(L.anc_run_batch_noalloc(len(arr), arr, C.c_void_p(stream)))
