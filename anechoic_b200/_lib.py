"""ctypes binding of libanechoic.so (the C ABI in include/anechoic.h).

The library is built in-tree (``python -m anechoic_b200.build_ext``). There is no fallback: if the library is missing
or CUDA is unavailable, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libanechoic.so")

ANC_OK, ANC_EINVAL, ANC_ECUDA, ANC_ETIMEOUT, ANC_EMISMATCH = 0, -1, -2, -3, -4
ENGINES = {"auto": 0, "plain": 1, "tensor": 2, "cluster": 3}
TENSOR_KINDS = {"auto": 0, "int8": 1, "fp4": 2}
KERNELS = {0: None, 1: "plain", 2: "tensor-int8", 3: "tensor-fp4", 4: "plain-cluster"}

EXPORTS = ("anc_instance_create", "anc_instance_create_csr", "anc_instance_get_info", "anc_instance_destroy",
           "anc_tables_create", "anc_tables_from_schedule", "anc_tables_steps", "anc_tables_read", "anc_tables_destroy",
           "anc_range_plan", "anc_schedule_tables", "anc_plan_ranges", "anc_spin_words", "anc_np", "anc_run",
           "anc_run_fields", "anc_run_device",
           "anc_run_batch", "anc_last_device_ms", "anc_last_kernel", "anc_last_error", "anc_last_profile", "anc_version",
           "anc_run_batch_noalloc", "anc_mf_create", "anc_mf_npad", "anc_mf_forward", "anc_mf_backward",
           "anc_mf_check", "anc_mf_set_wait_ns", "anc_mf_destroy", "anc_set_wait_ns", "anc_get_wait_ns",
           "anc_sparse_tuning", "anc_kernel_tuning")


class AncError(RuntimeError):
    """Error status from the C ABI (code is one of ANC_E*)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class InstanceInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("np", C.c_int), ("kbits", C.c_int), ("sparse", C.c_int), ("nnz", C.c_int64),
                ("sumw", C.c_int64), ("maxabs", C.c_int32), ("hmax", C.c_int64), ("bmax", C.c_int32),
                ("mean_row_sq", C.c_double)]


class RunOpts(C.Structure):
    _fields_ = [("engine", C.c_int), ("wide", C.c_int), ("threads", C.c_int), ("profile", C.c_int),
                ("tensor_kind", C.c_int), ("flip_permille", C.c_int), ("sparse_variant", C.c_int),
                ("kernel_variant", C.c_int)]


class Job(C.Structure):
    _fields_ = [("inst", C.c_void_p), ("tb", C.c_void_p), ("seed", C.c_uint64), ("trial_offset", C.c_uint32),
                ("nchains", C.c_int), ("spins", C.c_void_p), ("sum_sh", C.c_void_p), ("sum_bs", C.c_void_p),
                ("flips", C.c_void_p), ("trace", C.c_void_p)]


_lib = None
_lock = threading.Lock()

_vp, _i, _u32, _u64, _d = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_double


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: build it with `python -m anechoic_b200.build_ext`")
        L = C.CDLL(path)
        L.anc_instance_create.argtypes = [_vp, _i, _i, _vp, C.POINTER(_vp)]
        L.anc_instance_create_csr.argtypes = [_i, _vp, _vp, _vp, _vp, C.POINTER(_vp)]
        L.anc_instance_get_info.argtypes = [_vp, C.POINTER(InstanceInfo)]
        L.anc_instance_destroy.argtypes = [_vp]
        L.anc_instance_destroy.restype = None
        L.anc_tables_create.argtypes = [_vp, _vp, _vp, _vp, _i, C.POINTER(_vp)]
        L.anc_tables_from_schedule.argtypes = [_i, _d, _d, _d, _d, _d, _d, _i, _d, C.POINTER(_vp)]
        L.anc_tables_steps.argtypes = [_vp]
        L.anc_tables_read.argtypes = [_vp, _vp, _vp, _vp, _vp]
        L.anc_tables_destroy.argtypes = [_vp]
        L.anc_tables_destroy.restype = None
        L.anc_range_plan.argtypes = [_vp, _vp, C.POINTER(_i), C.POINTER(C.c_int32)]
        L.anc_schedule_tables.argtypes = [_i, _d, _d, _d, _d, _d, _d, _i, _d, _vp, _vp, _vp, _vp]
        L.anc_plan_ranges.argtypes = [_i, C.c_int64, C.c_int64, _vp, _vp, _vp, _vp, _i, C.POINTER(_i),
                                      C.POINTER(C.c_int32)]
        L.anc_spin_words.argtypes = [_i]
        L.anc_np.argtypes = [_i]
        L.anc_run.argtypes = [_vp, _vp, _u64, _u32, _i, C.POINTER(RunOpts), _vp, _vp, _vp, _vp, _vp]
        L.anc_run_fields.argtypes = [_vp, _vp, _u64, _u32, _i, C.POINTER(RunOpts), _vp, _vp, _vp, _vp, _vp, _vp]
        L.anc_run_device.argtypes = [_vp, _vp, _u64, _u32, _i, C.POINTER(RunOpts), _vp, _vp, _vp, _vp, _vp, _vp]
        L.anc_run_batch.argtypes = [_i, C.POINTER(Job), C.POINTER(RunOpts)]
        L.anc_auto_estimate.argtypes = [_i, _i, _i, _i, _d, _i, _vp, _vp]
        L.anc_auto_choice.argtypes = [_vp, _vp, _i, C.POINTER(RunOpts), _vp, _vp, _vp]
        L.anc_last_device_ms.argtypes = []
        L.anc_last_device_ms.restype = C.c_double
        L.anc_last_kernel.argtypes = []
        L.anc_last_kernel.restype = C.c_int
        L.anc_last_error.argtypes = []
        L.anc_last_error.restype = C.c_char_p
        L.anc_last_profile.argtypes = [C.POINTER(C.c_double), C.c_int]
        L.anc_version.argtypes = []
        L.anc_version.restype = C.c_char_p
        L.anc_set_wait_ns.argtypes = [_u64]
        L.anc_get_wait_ns.argtypes = []
        L.anc_get_wait_ns.restype = _u64
        L.anc_sparse_tuning.argtypes = [_vp, C.POINTER(_i), _vp]
        L.anc_kernel_tuning.argtypes = [_vp, _i, _i, C.POINTER(_i), C.POINTER(_i), _vp]
        _lib = L
        return L


def check(rc: int):
    if rc != ANC_OK:
        msg = load().anc_last_error().decode(errors="replace")
        raise AncError(rc, msg)


def opts(engine: str = "auto", wide="auto", profile: bool = False, tensor_kind: str = "auto",
         flip_fraction=None) -> RunOpts:
    o = RunOpts()
    o.engine = ENGINES[engine]
    o.tensor_kind = TENSOR_KINDS[tensor_kind]
    o.wide = {"auto": -1, 0: 0, 1: 1, False: 0, True: 1, "0": 0, "1": 1}[wide]
    o.threads = 0
    o.profile = int(bool(profile))
    o.flip_permille = 0 if flip_fraction is None else max(1, min(1000, int(round(1000 * flip_fraction))))
    return o


# Tensor-engine phase counters (SM cycles per step, averaged over CTAs). Names follow the fp4 kernel; the int8 and
# streaming kernels fill slots 2-7 with: named barrier + n_lin publish, cluster barrier, n_lin read, MMA waiting for
# TMA stages, MMA phase, TMA waiting for free stages.
PROFILE_FIELDS = ("wait_fields", "decide", "publish", "draw", "exchange", "mma_wait", "mma_phase", "tma_wait_stage",
                  "step", "ctas", "cluster", "max_active_clusters", "mma_issue", "mma_commit",
                  "first_tile_after_publish", "last_tile_after_publish", "nlin_tile_after_publish",
                  "fields_commit_after_publish", "tile0_flags_after_publish", "tile7_flags_after_publish",
                  "tile0_stored_after_publish", "tile7_stored_after_publish",
                  *(f"tile{t}_full_after_publish" for t in range(2, 7)),
                  *(f"warp{w}_tile7_stored_after_publish" for w in range(8)),
                  *(f"warp{w}_tile7_flags_after_publish" for w in range(8)),
                  *(f"tile{t}_issued_after_publish" for t in range(8)),
                  *(f"tile{t}_mma_wait" for t in range(8)))


def last_kernel():
    """Kernel of this thread's last single-instance run: "plain", "plain-cluster", "tensor-int8", "tensor-fp4" (None
    before any)."""
    return KERNELS[load().anc_last_kernel()]


def last_profile() -> dict:
    """Phase profile (SM cycles per step) of this thread's last profiled tensor-engine run."""
    buf = (C.c_double * len(PROFILE_FIELDS))()
    k = load().anc_last_profile(buf, len(PROFILE_FIELDS))
    return {PROFILE_FIELDS[i]: buf[i] for i in range(k)}
