"""TEST INFRASTRUCTURE ONLY: ctypes access to the two checkers.

* ``Restatement`` -- this project's C restatement of the golden model (oracle/sca_oracle.c, liboracle.so).
* ``Reference``   -- the reference's own golden model compiled unmodified (oracle/_ref/libscaref.so), present only where
  the reference tree was available at build time.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module. The product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libscaref.so")

_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def np_pad(n: int) -> int:
    """Padded spin count NP(n) = max(2048, ceil(n / 256) * 256)."""
    return max(2048, -(-n // 256) * 256)


class _Inst(C.Structure):
    _fields_ = [("n", C.c_int), ("dense", C.c_void_p), ("row_ptr", C.c_void_p), ("col", C.c_void_p),
                ("val", C.c_void_p), ("bias", C.c_void_p)]


class _Tab(C.Structure):
    _fields_ = [("fourT", C.c_void_p), ("q", C.c_void_p), ("kcorr", C.c_void_p), ("kconst", C.c_void_p), ("S", C.c_int)]


def _ptr(a):
    return None if a is None else a.ctypes.data


def build():
    """Compile liboracle.so (and oracle/_ref when the reference tree is present) with oracle/Makefile."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Restatement:
    """The C restatement. Instances are dense int8 (n x n, row-major) or CSR (row_ptr, col, val)."""

    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_np.argtypes = [C.c_int]
        L.orc_np.restype = C.c_int
        L.orc_tables.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int, C.c_double, _i32p, _i32p, _i64p, _i32p]
        L.orc_run.argtypes = [C.POINTER(_Inst), C.POINTER(_Tab), C.c_uint64, C.c_uint32, C.c_int, _u64p,
                              C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_void_p, C.c_void_p]
        L.orc_run_batch.argtypes = [C.POINTER(_Inst), C.POINTER(_Tab), C.c_uint64, C.c_uint32, C.c_int, C.c_int, C.c_int,
                                    _u64p, _i64p, _i64p, _i64p, C.c_void_p]

    def tables(self, S, t0=30.0, t1=5.0, q=4.0, lam=0.0, jv=0.0, kappa=0.0, ramp=False, scale=1.0):
        f = np.zeros(S, np.int32); qq = np.zeros(S, np.int32); kc = np.zeros(S, np.int64); ks = np.zeros(S, np.int32)
        if self.lib.orc_tables(S, t0, t1, q, lam, jv, kappa, int(bool(ramp)), scale, f, qq, kc, ks):
            raise ValueError("orc_tables failed")
        return dict(fourT=f, q=qq, kcorr=kc, kconst=ks)

    @staticmethod
    def _inst(n, dense=None, csr=None, bias=None):
        keep = []
        inst = _Inst()
        inst.n = n
        if dense is not None:
            d = np.ascontiguousarray(dense, np.int8)
            assert d.shape == (n, n)
            keep.append(d); inst.dense = _ptr(d)
        else:
            rp, col, val = (np.ascontiguousarray(csr[0], np.int32), np.ascontiguousarray(csr[1], np.int32),
                            np.ascontiguousarray(csr[2], np.int8))
            keep += [rp, col, val]
            inst.row_ptr, inst.col, inst.val = _ptr(rp), _ptr(col), _ptr(val)
        if bias is not None:
            b = np.ascontiguousarray(bias, np.int32)
            keep.append(b); inst.bias = _ptr(b)
        return inst, keep

    @staticmethod
    def _tab(tb):
        keep = [np.ascontiguousarray(tb["fourT"], np.int32), np.ascontiguousarray(tb["q"], np.int32),
                np.ascontiguousarray(tb["kcorr"], np.int64), np.ascontiguousarray(tb["kconst"], np.int32)]
        t = _Tab()
        t.fourT, t.q, t.kcorr, t.kconst = (_ptr(a) for a in keep)
        t.S = len(keep[0])
        return t, keep

    def run(self, n, tb, seed, trial, dense=None, csr=None, bias=None, trace=True, want_h=False):
        inst, k1 = self._inst(n, dense, csr, bias)
        tab, k2 = self._tab(tb)
        words = np_pad(n) // 64
        spins = np.zeros(words, np.uint64)
        sh, bs, fl = C.c_int64(), C.c_int64(), C.c_int64()
        nlin = np.zeros(tab.S, np.int32)
        h = np.zeros(n, np.int32) if want_h else None
        rc = self.lib.orc_run(C.byref(inst), C.byref(tab), seed, trial, int(trace), spins, C.byref(sh), C.byref(bs),
                              C.byref(fl), _ptr(nlin), _ptr(h))
        if rc:
            raise ValueError("orc_run failed")
        out = dict(spins=spins, sum_sh=sh.value, sum_bs=bs.value, flips=fl.value, nlin=nlin if trace else None)
        if want_h:
            out["h"] = h
        return out

    def run_batch(self, n, tb, seed, trial_offset, ntrials, dense=None, csr=None, bias=None, trace=True, threads=None):
        inst, k1 = self._inst(n, dense, csr, bias)
        tab, k2 = self._tab(tb)
        words = np_pad(n) // 64
        spins = np.zeros((ntrials, words), np.uint64)
        sh = np.zeros(ntrials, np.int64); bs = np.zeros(ntrials, np.int64); fl = np.zeros(ntrials, np.int64)
        nlin = np.zeros((ntrials, tab.S), np.int32) if trace else None
        th = threads or os.cpu_count() or 1
        rc = self.lib.orc_run_batch(C.byref(inst), C.byref(tab), seed, trial_offset, ntrials, int(trace), th,
                                    spins, sh, bs, fl, _ptr(nlin))
        if rc:
            raise ValueError("orc_run_batch failed")
        return dict(spins=spins, sum_sh=sh, sum_bs=bs, flips=fl, nlin=nlin)


class Reference:
    """The reference's golden model (NP = 2048, LANES = 256); dense matrices are passed as NP x NP int8."""

    NP = 2048

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_build_tables.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int, _i32p, _i32p, _i64p, _i32p]
        L.ref_mb_tables.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int, C.c_double, _i32p, _i32p, _i64p, _i32p]
        L.ref_run_trial_bias.argtypes = [C.c_int, _i8p, C.c_void_p, _i32p, _i32p, _i64p, _i32p, C.c_int, C.c_uint64,
                                         C.c_uint32, C.c_int, _u64p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int64), _i32p]
        L.ref_run_trial.argtypes = [_i8p, C.c_int64, _i32p, _i32p, _i64p, _i32p, C.c_int, C.c_uint64, C.c_uint32, C.c_int,
                                    _u64p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _i32p]
        L.ref_run_batch_bias.argtypes = [C.c_int, _i8p, C.c_void_p, _i32p, _i32p, _i64p, _i32p, C.c_int, C.c_uint64,
                                         C.c_uint32, C.c_int, C.c_int, C.c_int, _u64p, _i64p, _i64p, _i64p, _i32p]

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_LIB)

    def build_tables(self, S, t0=30.0, t1=5.0, q=4.0, lam=0.0, jv=0.0, kappa=0.0, ramp=False):
        f = np.zeros(S, np.int32); qq = np.zeros(S, np.int32); kc = np.zeros(S, np.int64); ks = np.zeros(S, np.int32)
        if self.lib.ref_build_tables(S, t0, t1, q, lam, jv, kappa, int(bool(ramp)), f, qq, kc, ks):
            raise ValueError("build_tables failed")
        return dict(fourT=f, q=qq, kcorr=kc, kconst=ks)

    def mb_tables(self, S, t0=30.0, t1=5.0, q=4.0, lam=0.0, jv=0.0, kappa=0.0, ramp=False, scale=1.0):
        f = np.zeros(S, np.int32); qq = np.zeros(S, np.int32); kc = np.zeros(S, np.int64); ks = np.zeros(S, np.int32)
        if self.lib.ref_mb_tables(S, t0, t1, q, lam, jv, kappa, int(bool(ramp)), scale, f, qq, kc, ks):
            raise ValueError("mb::tables failed")
        return dict(fourT=f, q=qq, kcorr=kc, kconst=ks)

    @classmethod
    def padded(cls, dense):
        n = dense.shape[0]
        d = np.zeros((cls.NP, cls.NP), np.int8)
        d[:n, :n] = dense
        return d

    def run_trial_bias(self, n, dense, bias, tb, seed, trial, trace=True):
        d = self.padded(dense)
        b = None if bias is None else np.ascontiguousarray(np.pad(np.asarray(bias, np.int32), (0, self.NP - n)))
        spins = np.zeros(32, np.uint64)
        sh, bs, fl = C.c_int64(), C.c_int64(), C.c_int64()
        S = len(tb["fourT"])
        nlin = np.zeros(S, np.int32)
        rc = self.lib.ref_run_trial_bias(n, d, _ptr(b), tb["fourT"], tb["q"], tb["kcorr"], tb["kconst"], S, seed, trial,
                                         int(trace), spins, C.byref(sh), C.byref(bs), C.byref(fl), nlin)
        if rc:
            raise ValueError("run_trial_bias failed")
        return dict(spins=spins, sum_sh=sh.value, sum_bs=bs.value, flips=fl.value, nlin=nlin if trace else None)

    def run_trial(self, dense, sumw, tb, seed, trial, trace=True):
        d = self.padded(dense)
        spins = np.zeros(32, np.uint64)
        cut, fl = C.c_int64(), C.c_int64()
        S = len(tb["fourT"])
        nlin = np.zeros(S, np.int32)
        rc = self.lib.ref_run_trial(d, sumw, tb["fourT"], tb["q"], tb["kcorr"], tb["kconst"], S, seed, trial, int(trace),
                                    spins, C.byref(cut), C.byref(fl), nlin)
        if rc:
            raise ValueError("run_trial failed")
        return dict(spins=spins, cut=cut.value, flips=fl.value, nlin=nlin if trace else None)

    def run_batch_bias(self, n, dense, bias, tb, seed, trial_offset, ntrials, trace=False, threads=None):
        d = self.padded(dense)
        b = None if bias is None else np.ascontiguousarray(np.pad(np.asarray(bias, np.int32), (0, self.NP - n)))
        S = len(tb["fourT"])
        spins = np.zeros((ntrials, 32), np.uint64)
        sh = np.zeros(ntrials, np.int64); bs = np.zeros(ntrials, np.int64); fl = np.zeros(ntrials, np.int64)
        nlin = np.zeros((ntrials, S), np.int32)
        th = threads or os.cpu_count() or 1
        rc = self.lib.ref_run_batch_bias(n, d, _ptr(b), tb["fourT"], tb["q"], tb["kcorr"], tb["kconst"], S, seed,
                                         trial_offset, ntrials, int(trace), th, spins, sh, bs, fl, nlin)
        if rc:
            raise ValueError("run_batch_bias failed")
        return dict(spins=spins, sum_sh=sh, sum_bs=bs, flips=fl, nlin=nlin if trace else None)
