"""ctypes binding of libaxr.so (include/axr.h).

There is no CPU fallback: if the library is missing or cannot be loaded,
`lib()` raises, and every draw call fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaxr.so")

# every symbol include/axr.h declares (tests check the exports against this)
EXPORTS = [
    "axr_last_error", "axr_create", "axr_destroy", "axr_set_scale_cull", "axr_add_texture_group",
    "axr_set_vert_light", "axr_vert_light", "axr_transform", "axr_translate", "axr_set_mip_bias", "axr_get_vertices",
    "axr_copy_to", "axr_ssao", "axr_dof", "axr_bloom", "axr_add_tex_alpha", "axr_set_primary_light",
    "axr_set_pos", "axr_set_vm", "axr_clear_zbuffer", "axr_draw_all", "axr_get_frame", "axr_get_ids",
    "axr_set_frame", "axr_gamma", "axr_add_shadow_map", "axr_place_shadow_map", "axr_clear_shadow_map",
    "axr_shadow_map", "axr_get_shadow_map", "axr_sync", "axr_get_stream", "axr_frame_device_ptrs",
    "axr_last_stats", "axr_launch_count", "axr_set_kernel_timing", "axr_kernel_times",
    "axr_shadow_map_noalloc", "axr_batch_create", "axr_batch_set_views", "axr_batch_render",
    "axr_batch_get_frame", "axr_batch_get_ids", "axr_batch_stats", "axr_batch_destroy",
    "axr_batch_set_tuning", "axr_set_tuning", "axr_batch_query", "axr_batch_read_async", "axr_batch_bytes",
    "axr_clear_color", "axr_batch_phase_times", "axr_batch_set_mode", "axr_read_frame_async", "axr_wait_frame",
    "axr_frame_done", "axr_batch_inject_barrier_stall", "axr_read_frame_rgb8_async", "axr_set_shadow_mode",
    "axr_shadow_stats", "axr_last_queues", "axr_add_normal_map", "axr_set_normal_material",
]


class ViewDesc(C.Structure):
    """axr_view_desc of include/axr.h"""
    _fields_ = [("kind", C.c_int), ("w", C.c_int), ("h", C.c_int), ("pos", C.c_float * 3), ("vm", C.c_float * 9),
                ("scale", C.c_float), ("cax", C.c_float), ("cay", C.c_float), ("bias", C.c_float),
                ("cascades", C.c_int * 2), ("ncascades", C.c_int), ("group_first", C.c_int),
                ("group_count", C.c_int), ("clear_color", C.c_int), ("bg", C.c_int * 3)]

vp = C.c_void_p
i32 = C.c_int
f32 = C.c_float

_SIGS = {
    "axr_last_error": (C.c_char_p, []),
    "axr_create": (i32, [i32, i32, i32, C.POINTER(vp)]),
    "axr_destroy": (i32, [vp]),
    "axr_set_scale_cull": (i32, [vp, f32, f32, f32]),
    "axr_add_texture_group": (i32, [vp, vp, vp, vp, i32, vp, vp, vp, C.c_long, i32, C.POINTER(i32)]),
    "axr_set_vert_light": (i32, [vp, i32, vp]),
    "axr_vert_light": (i32, [vp, vp, i32, vp, vp, i32, vp, vp, i32, vp, vp, vp, i32, f32]),
    "axr_transform": (i32, [vp, i32, vp, vp, vp, i32, i32]),
    "axr_translate": (i32, [vp, i32, vp, i32, i32]),
    "axr_get_vertices": (i32, [vp, i32, vp, vp, vp]),
    "axr_set_mip_bias": (i32, [vp, i32, f32]),
    "axr_ssao": (i32, [vp, vp, i32]),
    "axr_dof": (i32, [vp, f32]),
    "axr_bloom": (i32, [vp]),
    "axr_copy_to": (i32, [vp, i32, vp, vp, i32, i32]),
    "axr_add_tex_alpha": (i32, [vp, vp, i32, C.POINTER(i32)]),
    "axr_set_primary_light": (i32, [vp, vp, vp]),
    "axr_set_pos": (i32, [vp, vp]),
    "axr_set_vm": (i32, [vp, vp]),
    "axr_clear_zbuffer": (i32, [vp]),
    "axr_draw_all": (i32, [vp, vp, vp, vp, i32, vp, i32]),
    "axr_get_frame": (i32, [vp, vp, vp, vp, vp]),
    "axr_get_ids": (i32, [vp, vp, vp]),
    "axr_set_frame": (i32, [vp, vp, vp, vp, vp]),
    "axr_gamma": (i32, [vp, f32]),
    "axr_add_shadow_map": (i32, [vp, i32, i32, f32, f32]),
    "axr_place_shadow_map": (i32, [vp, i32, vp, vp, f32]),
    "axr_clear_shadow_map": (i32, [vp, i32]),
    "axr_shadow_map": (i32, [vp, i32, vp, vp, vp, i32, f32]),
    "axr_get_shadow_map": (i32, [vp, i32, vp]),
    "axr_sync": (i32, [vp]),
    "axr_get_stream": (i32, [vp, C.POINTER(vp)]),
    "axr_frame_device_ptrs": (i32, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "axr_last_stats": (i32, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                             C.POINTER(C.c_int64)]),
    "axr_launch_count": (i32, [vp, C.POINTER(C.c_int64)]),
    "axr_set_kernel_timing": (i32, [vp, i32]),
    "axr_kernel_times": (i32, [vp, i32, C.c_char_p, i32, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                               C.POINTER(i32)]),
    "axr_shadow_map_noalloc": (i32, [vp, vp, vp, i32, i32, vp, vp, f32, f32, vp, i32, vp]),
    "axr_batch_create": (i32, [vp, vp, i32, C.POINTER(vp)]),
    "axr_batch_set_views": (i32, [vp, vp, i32]),
    "axr_batch_render": (i32, [vp, vp, vp, vp, i32]),
    "axr_batch_get_frame": (i32, [vp, i32, vp, vp, vp, vp]),
    "axr_batch_get_ids": (i32, [vp, i32, vp, vp]),
    "axr_batch_stats": (i32, [vp, C.POINTER(C.c_int64), C.POINTER(i32), C.POINTER(i32)]),
    "axr_batch_destroy": (i32, [vp]),
    "axr_batch_set_tuning": (i32, [vp, i32, i32]),
    "axr_set_tuning": (i32, [vp, i32]),
    "axr_set_shadow_mode": (i32, [vp, i32, i32]),
    "axr_shadow_stats": (i32, [vp, i32, C.POINTER(C.c_int64), i32]),
    "axr_last_queues": (i32, [vp, C.POINTER(C.c_int64), i32]),
    "axr_add_normal_map": (i32, [vp, vp, C.c_long, C.POINTER(i32)]),
    "axr_set_normal_material": (i32, [vp, i32, i32, f32, i32]),
    "axr_batch_query": (i32, [vp]),
    "axr_batch_read_async": (i32, [vp, i32, vp, vp, vp, vp]),
    "axr_batch_bytes": (i32, [vp, C.POINTER(C.c_int64)]),
    "axr_clear_color": (i32, [vp, i32, i32, i32]),
    "axr_batch_phase_times": (i32, [vp, vp]),
    "axr_batch_set_mode": (i32, [vp, i32]),
    "axr_read_frame_async": (i32, [vp, vp, vp, vp, vp, C.POINTER(C.c_int64)]),
    "axr_wait_frame": (i32, [vp, C.c_int64]),
    "axr_frame_done": (i32, [vp, C.c_int64]),
    "axr_batch_inject_barrier_stall": (i32, [vp, i32, C.c_longlong]),
    "axr_read_frame_rgb8_async": (i32, [vp, f32, vp, C.POINTER(C.c_int64)]),
}

_lib = None


class AxrError(RuntimeError):
    pass


def lib():
    """Loads libaxr.so; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AxrError(f"{LIB_PATH} is not built: run `python -m axi_visualizer_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str):
    if rc != 0:
        msg = lib().axr_last_error().decode(errors="replace")
        raise AxrError(f"{what} failed ({rc}): {msg}")
