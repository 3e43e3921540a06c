"""ctypes binding of libpamo_b200.so (the C ABI in include/pamo_b200.h).

There is no fallback: if the library or a CUDA device is missing, every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpamo_b200.so")

PAMO_OK = 0
STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "out of device memory",
    3: "budget exceeded",
    4: "CUDA device error",
    5: "no CUDA device",
    6: "internal capacity exceeded",
}

# name -> (restype, argtypes); kept in step with include/pamo_b200.h
_vp, _i, _f, _ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_longlong
_ip = ctypes.POINTER(ctypes.c_int)
SIGNATURES = {
    "pamo_version": (_i, []),
    "pamo_launch_count": (_ll, []),
    "pamo_voronoi_areas": (_i, [_vp, _vp, _i, _i, _vp, ctypes.POINTER(ctypes.c_double), _vp]),
    "pamo_mesh_hinges": (_i, [_vp, _i, _i, _vp, _vp, ctypes.POINTER(ctypes.c_int)]),
    "pamo_mesh_hinges_device": (_i, [_vp, _i, _i, _vp, _vp, ctypes.POINTER(ctypes.c_int), _vp]),
    "pamo_merge_check_device": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_int), _vp]),
    "pamo_obj_parse": (_i, [_vp, _ll, _vp, _vp, _ll, _vp, _ll, _i, ctypes.POINTER(_ll), ctypes.POINTER(_ll),
                            ctypes.POINTER(_ll)]),
    "pamo_obj_format": (_i, [_vp, _ll, _vp, _ll, _vp, _ll, _i, ctypes.POINTER(_ll)]),
    "pamo_ply_parse": (_i, [_vp, _ll, _vp, _vp, _ll, _vp, _ll, ctypes.POINTER(_ll), ctypes.POINTER(_ll)]),
    "pamo_ply_format": (_i, [_vp, _ll, _vp, _ll, _vp, _ll, ctypes.POINTER(_ll)]),
    "pamo_point_stats": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_double), _vp]),
    "pamo_affine_points": (_i, [_vp, _i, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, _vp, _vp]),
    "pamo_batch_create": (_i, [_i, _ll, _ll, _i, _ll, _vp, ctypes.POINTER(_vp)]),
    "pamo_batch_destroy": (_i, [_vp]),
    "pamo_batch_submit": (_i, [_vp, _vp, _vp, _i, _i, _i, _ll, _i, _f, _i, ctypes.POINTER(_ll)]),
    "pamo_batch_step": (_i, [_vp, _ip, _ip]),
    "pamo_batch_job": (_i, [_vp, _ll, _ip, _ip, _ip, _ip]),
    "pamo_batch_finished": (_i, [_vp, ctypes.POINTER(_ll), _i]),
    "pamo_batch_fetch": (_i, [_vp, _ll, _vp, _vp, _i]),
    "pamo_batch_release": (_i, [_vp, _ll]),
    "pamo_batch_stats": (_i, [_vp, ctypes.POINTER(_ll)]),
    "pamo_batch_profile": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_ll), _i]),
    "pamo_status_string": (ctypes.c_char_p, [_i]),
    "pamo_ctx_create": (_i, [_i, ctypes.POINTER(_vp)]),
    "pamo_ctx_destroy": (_i, [_vp]),
    "pamo_free_forward": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _f, _f, _i, _i, _vp, _vp, _vp, _vp, _vp, _ip]),
    "pamo_free_copy_undo": (_i, [_vp, _vp, _i, _vp]),
    "pamo_stage2_run": (_i, [_vp, _vp, _vp, _i, _i, _ll, _i, _f, _i, _vp, _ip, _ip, _ip]),
    "pamo_stage2_fetch": (_i, [_vp, _vp, _vp, _i, _vp]),
    "pamo_set_quality": (_i, [_vp, _i]),
    "pamo_stage2_run_centred": (_i, [_vp, _vp, _vp, _i, _i, _vp, _ll, _i, _f, _i, _vp, _ip, _ip, _ip]),
    "pamo_remesh": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp, _ip, _ip]),
    "pamo_remesh_fetch": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "pamo_stage2_offset": (_i, [_vp, _vp]),
    "pamo_tris_mean": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "pamo_stage2_last_round_stats": (_i, [_vp, _vp]),
    "pamo_self_intersect": (_i, [_vp, _vp, _vp, _i, _i, _vp, ctypes.POINTER(_ll), _vp]),
    "pamo_profile_enable": (_i, [_vp, _i]),
    "pamo_profile_read": (_i, [_vp, _vp, _vp, _i]),
    "pamo_stage2_round_sizes": (_i, [_vp, _vp, _i]),
    "pamo_s3_default_config": (None, [_vp]),
    "pamo_safe_project": (_i, [_vp, _vp, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _i, _vp, _i, _vp, _i, _i, _vp, _vp,
                               _vp]),
    "pamo_safe_project_stats": (_i, [_vp, _vp]),
    "pamo_safe_project_trace": (_i, [_vp, _vp, _i, _ip]),
    "pamo_debug_wait_timeout": (_i, [_vp, _i, _ll, _vp]),
    "pamo_bsr_pcg": (_i, [_vp, _i, _vp, _vp, _vp, _ll, _vp, _vp, _i, _vp, _vp]),
    "pamo_self_intersect_noalloc": (_i, [_vp, _vp, _i, _i, _vp, ctypes.POINTER(_ll), _vp]),
    "pamo_check_mesh": (_i, [_vp, _vp, _i, _i, _vp, ctypes.POINTER(_ll), _vp]),
    "pamo_mesh_distance": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _i, _i, ctypes.POINTER(ctypes.c_double), _vp]),
    "pamo_simplify": (None, [_vp, _vp, _vp, _vp, _vp, _f]),
    "pamo_simplify_ctx": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _f]),
}

_lib = None


class PamoError(RuntimeError):
    def __init__(self, fn: str, code: int):
        super().__init__(f"{fn} failed: {STATUS.get(code, code)} ({code})")
        self.code = code


def lib():
    """Loads libpamo_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pamo_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(fn: str, code: int):
    if code != PAMO_OK:
        raise PamoError(fn, code)


PHASES = ["setup", "lbvh_build", "edge_cost", "collapse", "cleanup", "refit", "query", "pair_tests", "undo",
          "compact", "s3_closest", "s3_detect", "s3_diff", "s3_cg", "s3_ccd", "s3_line", "s1_prep", "s1_dist",
          "s1_flood", "s1_dmc"]


class Context:
    """Owns one pamo_ctx (device state carried between rounds)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        check("pamo_ctx_create", lib().pamo_ctx_create(int(device), ctypes.byref(self._h)))
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().pamo_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
