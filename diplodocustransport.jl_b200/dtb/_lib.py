"""ctypes binding of libdtb.so (the C ABI declared in include/dtb.h).

The library is built in-tree (diplodocustransport.jl_b200/lib/libdtb.so). There is no
fallback: if it is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libdtb.so")

DTB_OK, DTB_EINVAL, DTB_ENOMEM, DTB_ECUDA, DTB_ETIMEOUT, DTB_ESTATE, DTB_ENODEV, DTB_ENOTFOUND = range(8)
DTB_F64, DTB_F32, DTB_MIXED = 0, 1, 2
DTB_DTYPE_F64, DTB_DTYPE_F32 = 0, 1
DTB_FLAG_SYMPLECTIC = 1
DTB_FLAG_NO_AUTOTUNE = 2
DTB_FLUX_X, DTB_FLUX_P = 0, 1
MAX_SPECIES = 16

ERROR_NAMES = {1: "DTB_EINVAL", 2: "DTB_ENOMEM", 3: "DTB_ECUDA", 4: "DTB_ETIMEOUT", 5: "DTB_ESTATE",
               6: "DTB_ENODEV", 7: "DTB_ENOTFOUND"}


class DtbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Dims(ctypes.Structure):
    _fields_ = [("n_species", ctypes.c_int32), ("n_space", ctypes.c_int32),
                ("species_size", ctypes.c_int64 * MAX_SPECIES)]


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("device", ctypes.c_int32), ("stream", ctypes.c_void_p),
                ("index_base", ctypes.c_int32), ("graph_steps", ctypes.c_int32), ("dt0", ctypes.c_double),
                ("batch", ctypes.c_int32), ("flags", ctypes.c_int32)]


class ServeOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_int64), ("max_chunk_steps", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("chunk_ms", ctypes.c_double)]


class RequestStats(ctypes.Structure):
    _fields_ = [("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
                ("steps", ctypes.c_int64), ("cr_max", ctypes.c_double), ("finite", ctypes.c_int32),
                ("grid", ctypes.c_int32)]


class ServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("instance_steps", ctypes.c_int64), ("batched_steps", ctypes.c_int64),
                ("queued", ctypes.c_int64), ("running", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("busy_s", ctypes.c_double), ("elapsed_s", ctypes.c_double)]


class StepDiag(ctypes.Structure):
    _fields_ = [("cr", ctypes.c_double), ("cr_bin", ctypes.c_double), ("cr_emi", ctypes.c_double),
                ("cr_flux", ctypes.c_double), ("sum_df", ctypes.c_double), ("sum_f", ctypes.c_double),
                ("finite", ctypes.c_int32), ("pad", ctypes.c_int32)]


_P = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_d = ctypes.c_double

# name -> (restype, argtypes); every name is declared in include/dtb.h
SIGNATURES = {
    "dtb_abi_version": (_i32, []),
    "dtb_last_error": (ctypes.c_char_p, []),
    "dtb_device_count": (_i32, [_i32p]),
    "dtb_create": (_i32, [ctypes.POINTER(Dims), ctypes.POINTER(Opts), ctypes.POINTER(_P)]),
    "dtb_destroy": (_i32, [_P]),
    "dtb_add_flux_csc": (_i32, [_P, _i64, _ip, _ip, _dp]),
    "dtb_add_flux_csc_part": (_i32, [_P, _i32, _i64, _ip, _ip, _dp]),
    "dtb_upload_mbin_ref": (_i32, [_P, _dp, _i64]),
    "dtb_add_gain_block": (_i32, [_P, _i32, _i32, _i32, _P, _i32, _i32]),
    "dtb_add_loss_block": (_i32, [_P, _i32, _i32, _dp]),
    "dtb_upload_emi_ref": (_i32, [_P, _dp, _i64]),
    "dtb_add_emi_block": (_i32, [_P, _i64, _i64, _i64, _i64, _dp]),
    "dtb_upload_vectors": (_i32, [_P, _dp, _dp, _dp, _dp]),
    "dtb_set_bin_domain": (_i32, [_P, _ip, _i64]),
    "dtb_upload_mbin_csc": (_i32, [_P, _i64, _ip, _ip, _dp]),
    "dtb_commit": (_i32, [_P]),
    "dtb_step": (_i32, [_P, _d, _d, _d, _i32, _dp, _i32p, ctypes.POINTER(StepDiag)]),
    "dtb_step_io": (_i32, [_P, _dp, _dp, _d, _d, _d, _i32, _dp, _i32p, ctypes.POINTER(StepDiag)]),
    "dtb_run": (_i32, [_P, _dp, _i64, _i32, ctypes.POINTER(StepDiag)]),
    "dtb_solve": (_i32, [_P, _d, _dp, _i64, _i32, _dp, _ip]),
    "dtb_solve_ex": (_i32, [_P, _d, _dp, _i64, _i32, _dp, _dp, _dp, _dp, _ip]),
    "dtb_solve_schedule": (_i32, [_d, _dp, _i64, _d, _i32, _ip, _dp, _i64, _ip]),
    "dtb_get_f": (_i32, [_P, _dp]),
    "dtb_set_f": (_i32, [_P, _dp]),
    "dtb_reset": (_i32, [_P]),
    "dtb_moments": (_i32, [_P, _dp, _dp, _dp]),
    "dtb_device_bytes": (_i32, [_P, _ip]),
    "dtb_get_stream": (_i32, [_P, ctypes.POINTER(_P)]),
    "dtb_sync": (_i32, [_P]),
    "dtb_launches_per_step": (_i32, [_P, _i32p]),
    "dtb_launch_count": (_i32, [_P, _ip]),
    "dtb_gain_kernel_stats": (_i32, [_P, _dp, _dp]),
    "dtb_set_profiling": (_i32, [_P, _i32]),
    "dtb_selftest_bounded_wait": (_i32, [_P, _d]),
    "dtb_gain_contract": (_i32, [_i32, _P, _i64, _i64, _i64, _P, _P, _P, _P]),
    "dtb_gain_contract_status": (_i32, [_P]),
    "dtb_prepare": (_i32, [_P]),
    "dtb_selftest_gain_contract_timeout": (_i32, [_i32, _d, _P]),
    "dtb_batch_admit": (_i32, [_P, _i32, _dp, _d, _i64]),
    "dtb_batch_run": (_i32, [_P, _i64]),
    "dtb_batch_get_f": (_i32, [_P, _i32, _dp]),
    "dtb_batch_slot_info": (_i32, [_P, _i32, _ip, _ip, _dp, _i32p]),
    "dtb_batch_release": (_i32, [_P, _i32]),
    "dtb_batch_set_f_all": (_i32, [_P, _dp]),
    "dtb_batch_get_f_all": (_i32, [_P, _dp]),
    "dtb_batch_moments": (_i32, [_P, _dp, _dp, _dp]),
    "dtb_serve_create": (_i32, [ctypes.POINTER(ServeOpts), ctypes.POINTER(_P)]),
    "dtb_serve_add_grid": (_i32, [_P, _P, _i32p]),
    "dtb_serve_start": (_i32, [_P]),
    "dtb_serve_submit": (_i32, [_P, _i32, _dp, _d, _i64, _ip]),
    "dtb_serve_wait": (_i32, [_P, _i64, _d, _dp, ctypes.POINTER(RequestStats)]),
    "dtb_serve_cancel": (_i32, [_P, _i64]),
    "dtb_serve_get_stats": (_i32, [_P, ctypes.POINTER(ServeStats)]),
    "dtb_serve_destroy": (_i32, [_P]),
    "dtb_batch_capacity": (_i32, [_P, _i32p, _ip]),
    "dtb_batch_set_profiling": (_i32, [_P, _i32]),
    "dtb_batch_gemm_stats": (_i32, [_P, _dp, _dp, _dp, _i32p]),
    "dtb_set_tune_cache": (_i32, [ctypes.c_char_p]),
    "dtb_batch_run_io": (_i32, [_P, _P, _i64, _P]),
    "dtb_batch_gemm_plan": (_i32, [_P, _i32, _i32p, _i32p, _i32p, _dp]),
    "dtb_gain_contract_noalloc": (_i32, [_i32, _P, _i64, _i64, _i64, _P, _P, _P, _P]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libdtb.so and bind every declared entry point; raises if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libdtb.so not built: {path} is missing (run diplodocustransport.jl_b200/build.py)")
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != DTB_OK:
        msg = load().dtb_last_error()
        raise DtbError(rc, msg.decode() if msg else "")


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


class LastPtr:
    """dptr of the array passed last, kept while the same array object comes again: numpy's
    a.ctypes.data_as costs about 3 us a call, a visible share of a per-step host round trip.
    The array is referenced, so its buffer stays where the pointer points."""

    __slots__ = ("arr", "ptr")

    def __init__(self):
        self.arr = None
        self.ptr = None

    def __call__(self, a):
        if a is None:
            return None
        if a is not self.arr:
            self.arr, self.ptr = a, a.ctypes.data_as(_dp)
        return self.ptr


def iptr(a):
    return None if a is None else a.ctypes.data_as(_ip)
