"""ctypes binding of libhcfd_gpu.so (include/hcfd_gpu.h).

Loading fails loudly when the library is missing: there is no CPU fallback.  HCFD_LIB=checked
selects the checked twin libhcfd_gpu_checked.so (same entry points; its tile kernels verify
every index they read and report a bad one as HCFD_EINVAL instead of reading out of bounds).
"""
from __future__ import annotations

import ctypes as ct
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_DEFAULT = os.path.join(PKG, "lib", "libhcfd_gpu.so")
LIB_CHECKED = os.path.join(PKG, "lib", "libhcfd_gpu_checked.so")
_choice = os.environ.get("HCFD_LIB", "")
if _choice not in ("", "default", "checked"):
    raise RuntimeError(f"HCFD_LIB={_choice!r}: expected 'default' or 'checked'")
LIB_PATH = LIB_CHECKED if _choice == "checked" else LIB_DEFAULT

# status codes (include/hcfd_gpu.h)
OK, EINVAL, ENOMEM, ECUDA, ENONFINITE, ETIMEOUT, EIO, EAGAIN = 0, -1, -2, -3, -4, -5, -6, -7
# includes/Base/BoundaryConditions.hpp:6-13
SYMMETRY, WALL, SUPINLET, SUBINLET, SUPOUTLET, SUBOUTLET = range(6)
LIMITER_BJ, LIMITER_VENKAT = 0, 1
FIXED_DT, GLOBAL_CFL, LOCAL_CFL = 0, 1, 2
FP64, FP32 = 0, 1
NUMBER_NATURAL, NUMBER_RANDOM, NUMBER_RCM, NUMBER_MORTON = 0, 1, 2, 3
KERNEL_TILED, KERNEL_CELL = 0, 1

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)


class MeshView(ct.Structure):
    _fields_ = [("dim", ct.c_int), ("Nn", ct.c_int), ("Ncol", ct.c_int), ("NBCcol", ct.c_int),
                ("Nc", ct.c_int), ("Nf", ct.c_int),
                ("coltag", _ip), ("coloff", _ip), ("nodes", _dp), ("fn_con", _ip), ("fc_con", _ip),
                ("cn_off", _ip), ("cn_con", _ip), ("cc_off", _ip), ("cc_con", _ip)]


class WedgeSpec(ct.Structure):
    _fields_ = [("nx", ct.c_int), ("ny", ct.c_int), ("length", ct.c_double), ("height", ct.c_double),
                ("x_ramp", ct.c_double), ("theta_deg", ct.c_double), ("jitter", ct.c_double),
                ("seed", ct.c_uint64), ("numbering", ct.c_int)]


class Params(ct.Structure):
    _fields_ = [("gma", ct.c_double), ("limiter", ct.c_int), ("venkat_K", ct.c_double),
                ("precision", ct.c_int), ("block", ct.c_int), ("kernel", ct.c_int), ("tile", ct.c_int),
                ("keep_numbering", ct.c_int), ("freeze_limiter_after", ct.c_longlong), ("tile2", ct.c_int)]


class StepStats(ct.Structure):
    _fields_ = [("dt", ct.c_double), ("res_l2", ct.c_double), ("res_first", ct.c_double),
                ("steps", ct.c_longlong), ("nonfinite", ct.c_int)]


class ArenaParams(ct.Structure):
    _fields_ = [("hbm_budget", ct.c_size_t), ("precision", ct.c_int), ("limiter", ct.c_int),
                ("venkat_K", ct.c_double), ("gma", ct.c_double), ("time_mode", ct.c_int), ("tile", ct.c_int),
                ("slots", ct.c_int), ("max_instances", ct.c_int), ("freeze_limiter_after", ct.c_longlong)]


class ArenaInfo(ct.Structure):
    _fields_ = [("cell_capacity", ct.c_size_t), ("cells_used", ct.c_size_t), ("face_capacity", ct.c_size_t),
                ("faces_used", ct.c_size_t), ("active", ct.c_int), ("active_tiles", ct.c_int),
                ("steps", ct.c_longlong), ("tile", ct.c_int)]


class NoallocMesh(ct.Structure):
    _fields_ = [("Nc", ct.c_int), ("Nf", ct.c_int), ("F_BC", ct.c_int), ("slots", ct.c_int),
                ("slot", ct.c_void_p), ("geo", ct.c_void_p), ("iv", ct.c_void_p),
                ("nbc", ct.c_int), ("bc_first", _ip), ("bc_type", _ip), ("bc_state", _dp),
                ("gma", ct.c_double), ("limiter", ct.c_int), ("venkat_K", ct.c_double)]


NOALLOC_MAX_CELLS = 65536


class HcfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hcfd error {code}: {msg}")
        self.code = code


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "hcfd_mesh_load": (ct.c_int, [ct.c_char_p, ct.POINTER(ct.c_void_p)]),
    "hcfd_mesh_write": (ct.c_int, [ct.c_void_p, ct.c_char_p]),
    "hcfd_mesh_view_of": (ct.c_int, [ct.c_void_p, ct.POINTER(MeshView)]),
    "hcfd_mesh_cf": (ct.c_int, [ct.c_void_p, ct.POINTER(_ip), ct.POINTER(_ip)]),
    "hcfd_mesh_pname": (ct.c_char_p, [ct.c_void_p, ct.c_int]),
    "hcfd_mesh_free": (None, [ct.c_void_p]),
    "hcfd_mesh_generate_wedge": (ct.c_int, [ct.POINTER(WedgeSpec), ct.POINTER(ct.c_void_p)]),
    "hcfd_mesh_renumber": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_uint64]),
    "hcfd_gpu_create": (ct.c_int, [ct.POINTER(MeshView), ct.POINTER(Params), ct.POINTER(ct.c_void_p)]),
    "hcfd_gpu_gather_bcs": (ct.c_int, [ct.c_void_p, _ip, ct.c_int, _dp]),
    "hcfd_gpu_initialise": (ct.c_int, [ct.c_void_p, _dp]),
    "hcfd_gpu_step": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double, ct.POINTER(StepStats)]),
    "hcfd_gpu_download": (ct.c_int, [ct.c_void_p, ct.c_int, ct.POINTER(_dp)]),
    "hcfd_gpu_upload": (ct.c_int, [ct.c_void_p, ct.POINTER(_dp)]),
    "hcfd_gpu_sync": (ct.c_int, [ct.c_void_p]),
    "hcfd_gpu_stats": (ct.c_int, [ct.c_void_p, ct.POINTER(StepStats)]),
    "hcfd_gpu_test_waits": (ct.c_int, [ct.c_void_p, ct.c_uint, ct.c_int]),
    "hcfd_gpu_wall_cp": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double, ct.c_double, ct.c_double, _dp, _ip]),
    "hcfd_gpu_info": (ct.c_int, [ct.c_void_p, _ip, _ip, _ip, _ip]),
    "hcfd_gpu_profile": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "hcfd_gpu_profile_read": (ct.c_int, [ct.c_void_p, _dp, ct.POINTER(ct.c_longlong), _dp, ct.POINTER(ct.c_longlong)]),
    "hcfd_gpu_step_timed": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double, _dp]),
    "hcfd_gpu_launches_per_step": (ct.c_int, [ct.c_void_p]),
    "hcfd_gpu_destroy": (None, [ct.c_void_p]),
    "hcfd_host_pin": (ct.c_int, [ct.c_void_p, ct.c_size_t]),
    "hcfd_host_unpin": (ct.c_int, [ct.c_void_p]),
    "hcfd_write_hsln": (ct.c_int, [ct.c_char_p, ct.c_int, ct.POINTER(ct.c_char_p), ct.c_int, ct.POINTER(_dp)]),
    "hcfd_plan_check": (ct.c_int, [ct.POINTER(MeshView), ct.c_int, ct.c_int, ct.POINTER(ct.c_longlong)]),
    "hcfd_step_noalloc": (ct.c_int, [ct.POINTER(NoallocMesh), ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_double,
                                     ct.c_void_p, _dp, _dp]),
    "hcfd_gpu_snapshot": (ct.c_int, [ct.c_void_p, ct.c_int, ct.POINTER(_dp), ct.POINTER(ct.c_void_p)]),
    "hcfd_snapshot_wait": (ct.c_int, [ct.c_void_p]),
    "hcfd_snapshot_free": (None, [ct.c_void_p]),
    "hcfd_gpu_checkpoint": (ct.c_int, [ct.c_void_p, ct.c_char_p]),
    "hcfd_gpu_restore": (ct.c_int, [ct.c_void_p, ct.c_char_p]),
    "hcfd_checkpoint_info": (ct.c_int, [ct.c_char_p, _ip, _ip, ct.POINTER(ct.c_longlong), _ip]),
    "hcfd_arena_checkpoint": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_char_p]),
    "hcfd_arena_restore": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_char_p]),
    "hcfd_arena_create": (ct.c_int, [ct.POINTER(ArenaParams), ct.POINTER(ct.c_void_p)]),
    "hcfd_arena_admit": (ct.c_int, [ct.c_void_p, ct.POINTER(MeshView), _ip, ct.c_int, _dp, _dp, ct.c_double, _ip]),
    "hcfd_arena_prepare": (ct.c_int, [ct.c_void_p, ct.POINTER(MeshView), _ip, ct.c_int, _dp, _dp, ct.c_double,
                                      ct.POINTER(ct.c_void_p)]),
    "hcfd_arena_admit_prepared": (ct.c_int, [ct.c_void_p, ct.c_void_p, _ip]),
    "hcfd_admission_cells": (ct.c_size_t, [ct.c_void_p]),
    "hcfd_admission_free": (None, [ct.c_void_p]),
    "hcfd_arena_step": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "hcfd_arena_poll": (ct.c_int, [ct.c_void_p, ct.c_int, _ip, ct.POINTER(StepStats), _ip]),
    "hcfd_arena_fetch": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.POINTER(_dp)]),
    "hcfd_arena_release": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "hcfd_arena_info": (ct.c_int, [ct.c_void_p, ct.POINTER(ArenaInfo)]),
    "hcfd_arena_destroy": (None, [ct.c_void_p]),
    "hcfd_set_device": (ct.c_int, [ct.c_int, _ip]),
    "hcfd_device_sync": (ct.c_int, []),
    "hcfd_device_mem_info": (ct.c_int, [ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_size_t)]),
    "hcfd_last_error": (ct.c_char_p, []),
}


def lib():
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"native library missing: {LIB_PATH}; build it with "
                               f"`python -m cfd_optimisations_b200._build` (there is no CPU fallback)")
        L = ct.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc != OK:
        msg = lib().hcfd_last_error()
        raise HcfdError(rc, msg.decode() if msg else "")
    return rc
