"""Loader and ctypes prototypes of libspt_cuda.so, the C-ABI declared in include/spt.h.

There is no fallback: if the library is missing or cannot load, every entry point raises.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspt_cuda.so")

vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int32

# name -> (restype, argtypes); every function declared in include/spt.h
PROTOTYPES = {
    "spt_abi_version": (u32, []),
    "spt_create": (i32, [i32, C.POINTER(vp)]),
    "spt_destroy": (i32, [vp]),
    "spt_last_error": (C.c_char_p, [vp]),
    "spt_bvh_build": (i32, [vp, i32, C.POINTER(vp)]),
    "spt_bvh_build_device": (i32, [vp, vp, C.POINTER(vp)]),
    "spt_bvh_stats_get": (i32, [vp, vp]),
    "spt_bvh_export": (i32, [vp, vp, vp, vp, vp]),
    "spt_bvh_free": (i32, [vp]),
    "spt_scene_create": (i32, [vp, vp, vp, C.POINTER(vp)]),
    "spt_scene_destroy": (i32, [vp]),
    "spt_scene_device_bytes": (u64, [vp]),
    "spt_intersect": (i32, [vp, vp, vp, u64, vp, vp, vp]),
    "spt_intersect_packed": (i32, [vp, vp, vp, u64, vp, vp, vp]),
    "spt_intersect_device": (i32, [vp, vp, vp, u64, vp, vp]),
    "spt_ray_order_device": (i32, [vp, vp, vp, u64, vp, vp]),
    "spt_intersect_ordered_device": (i32, [vp, vp, vp, vp, u64, vp, vp]),
    "spt_hits_unorder_device": (i32, [vp, vp, u64, vp, vp, vp]),
    "spt_count_device": (i32, [vp, vp, vp, u64, vp, vp, vp, vp, vp]),
    "spt_traversal_work_device": (i32, [vp, vp, vp, u64, vp, vp]),
    "spt_intersect_noalloc": (i32, [vp, vp, vp, u64, vp, vp, vp]),
    "spt_raycast_image": (i32, [vp, vp, vp, i32, vp, vp]),
    "spt_raycast_image_device": (i32, [vp, vp, vp, i32, vp, vp]),
    "spt_pathtrace": (i32, [vp, vp, vp, vp, vp, vp]),
    "spt_pathtrace_device": (i32, [vp, vp, vp, vp, vp, vp]),
    "spt_write_ppm": (i32, [C.c_char_p, vp, u32, u32, i32]),
    "spt_depth_to_rgb_device": (i32, [vp, vp, u32, u32, C.c_float, C.c_float, vp, vp]),
    "spt_count_to_rgb_device": (i32, [vp, vp, u32, u32, C.c_int64, C.c_int64, vp, vp]),
    "spt_normal_to_rgb_device": (i32, [vp, vp, u32, u32, vp]),
    "spt_rgb_to_bytes_device": (i32, [vp, vp, u64, i32, vp, vp]),
    "spt_write_ppm_bytes": (i32, [C.c_char_p, vp, u32, u32]),
    "spt_tune_default": (i32, [vp]),
    "spt_batch_pathtrace": (i32, [vp, vp, u32, vp, vp, vp]),
    "spt_autotune": (i32, [vp, vp, u32, C.c_char_p, vp]),
    "spt_guide_create": (i32, [vp, vp, C.POINTER(vp)]),
    "spt_guide_destroy": (i32, [vp]),
    "spt_guide_get_params": (i32, [vp, vp, vp]),
    "spt_guide_set_params": (i32, [vp, vp, vp]),
    "spt_guide_eval": (i32, [vp, vp, vp, u32, vp]),
    "spt_guide_gradients": (i32, [vp, vp, vp, u32, vp, vp, vp]),
    "spt_guide_train": (i32, [vp, vp, vp, u32, vp]),
    "spt_guide_train_device": (i32, [vp, vp, vp, u32, C.POINTER(C.c_float)]),
    "spt_guide_steps": (i32, [vp, C.POINTER(C.c_uint64)]),
    "spt_guided_pathtrace_device": (i32, [vp, vp, vp, vp, vp, vp, vp]),
}

_lib = None


class SptError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (abi.STATUS_NAMES.get(status, str(status)), message))
        self.status = status


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libspt_cuda.so is not built (run __graft_entry__.build() or make -C "
                              "swpathtracer_b200/csrc): %s" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.spt_abi_version() != abi.SPT_ABI_VERSION:
            raise ImportError("libspt_cuda.so ABI version mismatch")
        _lib = L
    return _lib


def check(status, ctx=None, what=""):
    if status != abi.SPT_OK:
        msg = lib().spt_last_error(ctx).decode() if ctx else ""
        raise SptError(status, (what + ": " if what else "") + msg)
