"""ctypes binding of libbvhcuda's C ABI (include/bvhcuda.h).

Loading fails loudly: there is no Python or CPU fallback for any query.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libbvhcuda.so"

BVHC_OK = 0
FRONT_SIDE, BACK_SIDE, DOUBLE_SIDE = 0, 1, 2
CENTER, AVERAGE, SAH = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
NO_HIT = 0xFFFFFFFF


class BvhcHit(C.Structure):
    _fields_ = [("face_index", C.c_uint32), ("distance", C.c_float), ("point", C.c_float * 3),
                ("barycoord", C.c_float * 3)]


class BvhcClosest(C.Structure):
    _fields_ = [("face_index", C.c_uint32), ("distance", C.c_float), ("point", C.c_float * 3)]


class BvhcHitPointInfo(C.Structure):
    _fields_ = [("a", C.c_uint32), ("b", C.c_uint32), ("c", C.c_uint32), ("material_index", C.c_uint32),
                ("normal", C.c_float * 3), ("barycoord", C.c_float * 3), ("uv", C.c_float * 2)]


class BvhcTraversalConfig(C.Structure):
    _fields_ = [("persistent", C.c_int32), ("order", C.c_int32), ("refill", C.c_int32), ("occupancy", C.c_int32),
                ("compact", C.c_int32), ("sort", C.c_int32), ("closest", C.c_int32),
                ("wide", C.c_int32), ("all", C.c_int32), ("tile", C.c_int32),
                ("block", C.c_int32), ("stack", C.c_int32), ("tile_rows", C.c_int32)]


class BvhcMeshInfo(C.Structure):
    _fields_ = [("node_records", C.c_uint64), ("triangle_records", C.c_uint64), ("device_bytes", C.c_uint64),
                ("max_depth", C.c_int32), ("root_count", C.c_int32)]


# (name, restype, argtypes) for every entry point declared in include/bvhcuda.h
_P, _U64, _I64, _I, _F = C.c_void_p, C.c_uint64, C.c_int64, C.c_int, C.c_float
SIGNATURES = [
    ("bvhc_status_string", C.c_char_p, [_I]),
    ("bvhc_build", _I, [_P, _U64, _I, _P, _I, _U64, _P, _I, _I64, _I64, _I, _I, _I, _I, C.POINTER(_P)]),
    ("bvhc_build_device", _I, [_P, _U64, _I, _P, _I, _U64, _P, _I, _I64, _I64, _I, _I, _I, _I, _I, _P, C.POINTER(_P)]),
    ("bvhc_serialized_root_count", _I, [_P]),
    ("bvhc_serialized_root", _I, [_P, _I, C.POINTER(_P), C.POINTER(_U64)]),
    ("bvhc_serialized_index", _I, [_P, C.POINTER(_P), C.POINTER(_I), C.POINTER(_U64)]),
    ("bvhc_serialized_indirect", _I, [_P, C.POINTER(_P), C.POINTER(_I), C.POINTER(_U64)]),
    ("bvhc_serialized_free", None, [_P]),
    ("bvhc_mesh_create", _I, [_I, _I, _P, _P, _I, _P, _I, _U64, _P, _I, _U64, _P, _U64, _I, C.POINTER(_P)]),
    ("bvhc_mesh_destroy", None, [_P]),
    ("bvhc_mesh_get_info", _I, [_P, C.POINTER(BvhcMeshInfo)]),
    ("bvhc_mesh_synchronize", _I, [_P, _P]),
    ("bvhc_raycast_first", _I, [_P, _P, _U64, _I, _F, _F, _P, _I, _P]),
    ("bvhc_raycast", _I, [_P, _P, _U64, _I, _F, _F, C.c_uint32, _P, _P, _I, _P]),
    ("bvhc_closest_point_to_point", _I, [_P, _P, _U64, _F, _F, _P, _I, _P]),
    ("bvhc_mesh_set_groups", _I, [_P, _P, _I]),
    ("bvhc_batch_create", _I, [_I, _I, _P, _P, _P, _P, _I, _U64, _P, _U64, _I, C.POINTER(_P)]),
    ("bvhc_batch_mesh_count", _I, [_P]),
    ("bvhc_batch_raycast_first", _I, [_P, _P, _P, _I, _F, _F, _P, _P]),
    ("bvhc_batch_raycast_first_per_mesh", _I, [_P, _P, _P, _I, _F, _F, _P, _P]),
    ("bvhc_batch_graph_create", _I, [_P, _P, _P, _I, _F, _F, _P, C.POINTER(_P)]),
    ("bvhc_graph_launch", _I, [_P, _P]),
    ("bvhc_graph_destroy", None, [_P]),
    ("bvhc_mesh_enable_gradients", _I, [_P, _P, _I, _U64, _P, _U64, _I]),
    ("bvhc_raycast_first_backward", _I, [_P, _P, _P, _U64, _P, _P, _P, _P, _P, _P]),
    ("bvhc_closest_point_backward", _I, [_P, _P, _P, _U64, _P, _P, _P, _P]),
    ("bvhc_raycast_first_noalloc", _I, [_P, _P, _U64, _I, _F, _F, _P, _I, _P]),
    ("bvhc_mesh_set_traversal", _I, [_P, C.POINTER(BvhcTraversalConfig)]),
    ("bvhc_mesh_get_traversal", _I, [_P, C.POINTER(BvhcTraversalConfig)]),
    ("bvhc_mesh_set_leaf_size", _I, [_P, C.c_int]),
    ("bvhc_mesh_get_leaf_size", C.c_int, [_P]),
    ("bvhc_mesh_refit", _I, [_P, _P, C.c_uint64, C.c_int, C.c_int, _P]),
    ("bvhc_mesh_root_count", C.c_int, [_P]),
    ("bvhc_mesh_root_bytes", C.c_uint64, [_P, C.c_int]),
    ("bvhc_mesh_read_root", _I, [_P, C.c_int, _P, C.c_uint64]),
    ("bvhc_intersects_sphere", _I, [_P, _P, _U64, _P, _I, _P]),
    ("bvhc_intersects_box", _I, [_P, _P, _U64, _P, _I, _P]),
    ("bvhc_sphere_triangles", _I, [_P, _P, _U64, C.c_uint32, _P, _P, _I, _P]),
    ("bvhc_scene_create", _I, [_P, _I, _P, _P, _P, C.POINTER(_P)]),
    ("bvhc_scene_set_instances", _I, [_P, _I, _P, _P, _P]),
    ("bvhc_scene_raycast_first", _I, [_P, _P, _U64, _I, _F, _F, _P, _P, _I, _P]),
    ("bvhc_scene_destroy", None, [_P]),
    ("bvhc_scene_set_order", _I, [_P, _I]),
    ("bvhc_scene_set_variant", _I, [_P, _I]),
    ("bvhc_scene_raycast", _I, [_P, _P, _U64, _I, _F, _F, C.c_uint32, _P, _P, _P, _I, _P]),
    ("bvhc_hit_interpolate", _I, [_P, _P, _U64, _P, _U64, _I, _I, _P, _P, _I, _P]),
    ("bvhc_triangle_hit_point_info", _I, [_P, _P, _P, _U64, _P, _I, _P, _I, _U64, _P, _I, _P, _I, _P]),
    ("bvhc_raycast_first_materials", _I, [_P, _P, _U64, _P, _I, _F, _F, _P, _I, _P]),
    ("bvhc_raycast_materials", _I, [_P, _P, _U64, _P, _I, _F, _F, C.c_uint32, _P, _P, _I, _P]),
    ("bvhc_mesh_autotune", _I, [_P, _I, _P, _P, _I, _F, _F, _P, _I, _P, _I, _I, _P, C.POINTER(BvhcTraversalConfig),
                                _P, _P, _P]),
    ("bvhc_autotune_candidates", _I, [_P, _I, C.POINTER(BvhcTraversalConfig), _I]),
]

_lib = None


class BVHCError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().bvhc_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def lib() -> C.CDLL:
    """Load libbvhcuda.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"libbvhcuda.so not found at {LIB_PATH}; build it with __graft_entry__.build()")
        dll = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(dll, name)
            fn.restype = res
            fn.argtypes = args
        _lib = dll
    return _lib


def check(status: int, where: str) -> None:
    if status != BVHC_OK:
        raise BVHCError(status, where)
