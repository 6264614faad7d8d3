"""ctypes binding of libvoxrt (include/voxrt.h).

The shared library is built in-tree (python -m voxelg_b200.build) to
voxelg_b200/lib/libvoxrt.so.  There is no fallback: importing the traversal
API without the library raises, and every traversal call fails with
VX_ERR_CUDA when no GPU is usable.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

# VOXRT_CHECKED=1 loads the checked library (every world load bounds-checked,
# see vx_world_oob) instead of libvoxrt.so.
LIB_PATH = Path(__file__).resolve().parent / "lib" / (
    "libvoxrt_checked.so" if os.environ.get("VOXRT_CHECKED") == "1" else "libvoxrt.so")

VX_OK = 0
VX_ERR_INVALID = -1
VX_ERR_CUDA = -2
VX_ERR_OOM = -3
VX_ERR_DEVICE = -4
VX_ERR_BUSY = -5

VX_F_L4 = 1 << 0
VX_F_LUT = 1 << 1
VX_F_LOD = 1 << 2
VX_F_BEAM = 1 << 3
VX_F_SHADOW = 1 << 4
VX_F_METHOD = VX_F_L4 | VX_F_LUT | VX_F_LOD | VX_F_BEAM
VX_RAY_SPAWN_SHADOW = 1 << 8
VX_SERVE_SLOTS = 0
VX_SERVE_RESIDENT = 1


class VxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"voxrt error {code}: {msg}")
        self.code = code


class VxWorldDesc(C.Structure):
    _fields_ = [("bricks_x", C.c_int32), ("bricks_y", C.c_int32), ("bricks_z", C.c_int32),
                ("device", C.c_int32)]


class VxCamera(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("tan_half_fov", C.c_float), ("res_x", C.c_float),
                ("res_y", C.c_float), ("jitter_x", C.c_float), ("jitter_y", C.c_float),
                ("world_origin", C.c_int32 * 3)]


class VxTraceParams(C.Structure):
    _fields_ = [("max_dist", C.c_float), ("lod_brick_t", C.c_float), ("tile_lod_t", C.c_float),
                ("shadow_max_dist", C.c_float), ("beam_margin", C.c_float),
                ("max_iters", C.c_int32), ("any_max_iters", C.c_int32), ("flags", C.c_uint32),
                ("sun", C.c_float * 3), ("sun_tangent", C.c_float * 3),
                ("sun_bitangent", C.c_float * 3), ("cone_tan", C.c_float), ("frame", C.c_float)]


class VxPickHit(C.Structure):
    _fields_ = [("voxel", C.c_int32 * 3), ("normal", C.c_int32 * 3)]


class VxWorldView(C.Structure):
    _fields_ = [("bricks_x", C.c_int32), ("bricks_y", C.c_int32), ("bricks_z", C.c_int32),
                ("occupancy", C.c_void_p), ("materials", C.c_void_p), ("tile_mask", C.c_void_p),
                ("chunk_mask", C.c_void_p), ("l4_mask", C.c_void_p),
                ("brick_uniform", C.c_void_p), ("tile_uniform", C.c_void_p)]


class VxTuning(C.Structure):
    _fields_ = [("persistent", C.c_int32), ("reserved", C.c_int32 * 7)]


class VxQueueTuning(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("refill_min", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("sort", C.c_int32), ("reserved", C.c_int32 * 4)]


class VxServeConfig(C.Structure):
    _fields_ = [("mem_budget_bytes", C.c_uint64), ("slots", C.c_int32),
                ("max_batch_rays", C.c_int32), ("max_batch_requests", C.c_int32),
                ("mode", C.c_int32), ("idle_us", C.c_int32), ("wait_us", C.c_int32)]


class VxServeStats(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("rays", C.c_uint64), ("batches", C.c_uint64),
                ("rejected", C.c_uint64), ("edits", C.c_uint64), ("edited_bricks", C.c_uint64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("seconds", C.c_double), ("mrays_per_s", C.c_double),
                ("peak_inflight_rays", C.c_uint64)]


class VxServeLoad(C.Structure):
    _fields_ = [("clients", C.c_int32), ("rate_per_client", C.c_float), ("seconds", C.c_float),
                ("min_rays", C.c_int32), ("max_rays", C.c_int32), ("min_len", C.c_float),
                ("max_len", C.c_float), ("edit_fraction_per_s", C.c_float), ("seed", C.c_uint64)]


class VxTrainConfig(C.Structure):
    _fields_ = [("poses", C.c_uint32), ("rays_per_pose", C.c_uint32), ("steps", C.c_uint32),
                ("batch", C.c_uint32), ("lr", C.c_float), ("y_min", C.c_float),
                ("y_max", C.c_float), ("pitch_min", C.c_float), ("pitch_max", C.c_float),
                ("fov_y", C.c_float), ("width", C.c_uint32), ("height", C.c_uint32),
                ("flags", C.c_uint32), ("held_out_poses", C.c_uint32), ("seed", C.c_uint64)]


class VxLearnedStats(C.Structure):
    _fields_ = [("none", C.c_uint64), ("partial", C.c_uint64), ("accepted", C.c_uint64),
                ("miss", C.c_uint64), ("cells", C.c_uint64), ("iters", C.c_uint64),
                ("fallback", C.c_uint64), ("rays", C.c_uint64), ("infer_ms", C.c_float),
                ("trace_ms", C.c_float)]


MLP_FLOATS = 13569
MLP_FEATURES = 80


class VxTerrainParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("base_height", C.c_float), ("amplitude", C.c_float),
                ("inv_wavelength", C.c_float), ("octaves", C.c_uint32),
                ("water_level", C.c_int32), ("cave_inv_wavelength", C.c_float),
                ("cave_threshold", C.c_float), ("dirt_depth", C.c_int32)]


# numpy views of the record / brick layouts (byte-identical to voxrt.h)
BRICK_DTYPE = np.dtype([("occupancy", "<u8"), ("materials", "u1", (64,))])
RECORD_DTYPE = np.dtype([("voxel", "<i4", (3,)), ("face", "u1"), ("mat", "u1"), ("flags", "u1"),
                         ("pad", "u1"), ("t", "<f4"), ("steps", "<u4")])
SHADOW_DTYPE = np.dtype([("steps", "<u4"), ("occluded", "u1"), ("traced", "u1"), ("pad", "<u2")])
RAY_DTYPE = np.dtype([("org", "<f4", (3,)), ("dir", "<f4", (3,)), ("tmax", "<f4"),
                      ("kind", "<u4")])
PICK_DTYPE = np.dtype([("voxel", "<i4", (3,)), ("normal", "<i4", (3,))])
PACKED_DTYPE = np.dtype([("voxel", "<u4"), ("face", "u1"), ("mat", "u1"), ("flags", "u1"),
                         ("shadow", "u1"), ("t", "<f4"), ("steps", "<u4")])
assert BRICK_DTYPE.itemsize == 72 and RECORD_DTYPE.itemsize == 24
assert SHADOW_DTYPE.itemsize == 8 and RAY_DTYPE.itemsize == 32
assert PACKED_DTYPE.itemsize == 16
COMPACT_DTYPE = np.dtype([("w", "<u4", (3,))])
assert COMPACT_DTYPE.itemsize == 12

# every symbol include/voxrt.h declares: (name, restype, argtypes)
_vp = C.c_void_p
_P = C.POINTER
SIGNATURES = [
    ("vx_abi_version", C.c_int, []),
    ("vx_last_error", C.c_char_p, []),
    ("vx_default_params", C.c_int, [_P(VxTraceParams)]),
    ("vx_camera_from_pose", C.c_int, [_P(C.c_float), C.c_float, C.c_float, C.c_float, C.c_uint32,
                                      C.c_uint32, _P(C.c_int32), _P(VxCamera)]),
    ("vx_world_create", C.c_int, [_P(VxWorldDesc), _P(_vp)]),
    ("vx_world_destroy", C.c_int, [_vp]),
    ("vx_world_upload", C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("vx_world_download", C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("vx_world_generate", C.c_int, [_vp, _P(VxTerrainParams)]),
    ("vx_world_gen_chunks", C.c_int, [_vp, C.c_uint64, _vp, C.c_uint32]),
    ("vx_world_fill_window", C.c_int, [_vp, C.c_uint64, C.c_int32, C.c_int32]),
    ("vx_world_shift_origin", C.c_int, [_vp, C.c_int32, C.c_int32, _P(C.c_uint32)]),
    ("vx_world_apply_edit", C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_uint8]),
    ("vx_world_clear_edits", C.c_int, [_vp]),
    ("vx_world_save", C.c_int, [_vp, C.c_char_p]),
    ("vx_world_load", C.c_int, [_vp, C.c_char_p]),
    ("vx_world_apply_dirty", C.c_int, [_vp, _vp, _vp, C.c_size_t, _vp]),
    ("vx_world_counts", C.c_int, [_vp, _P(C.c_uint64)]),
    ("vx_checked_build", C.c_int, []),
    ("vx_render_primary_rows", C.c_int, [_vp, _vp, _vp, C.c_uint32, C.c_uint32, _vp, _vp, _vp]),
    ("vx_world_oob", C.c_int, [_vp, _P(C.c_uint64), C.c_int32]),
    ("vx_world_set_tuning", C.c_int, [_vp, _P(VxTuning)]),
    ("vx_world_get_tuning", C.c_int, [_vp, _P(VxTuning)]),
    ("vx_raycast", C.c_int, [_vp, _P(C.c_float), _P(C.c_float), _P(C.c_int32), _P(VxPickHit)]),
    ("vx_raycast_batch", C.c_int, [_vp, _P(C.c_int32), _vp, _vp, C.c_size_t, _vp, _vp, _vp]),
    ("vx_trace", C.c_int, [_vp, _P(C.c_int32), _vp, C.c_size_t, _P(VxTraceParams), _vp, _vp]),
    ("vx_render_primary", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp, _vp, _vp]),
    ("vx_render_primary_host", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp, _vp]),
    ("vx_render_primary_host_async", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp, _vp]),
    ("vx_render_host_wait", C.c_int, [_vp]),
    ("vx_render_primary_host_packed", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp]),
    ("vx_render_primary_host_packed_async", C.c_int,
     [_vp, _P(VxCamera), _P(VxTraceParams), _vp]),
    ("vx_render_primary_host_compact", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp]),
    ("vx_render_primary_host_compact_async", C.c_int,
     [_vp, _P(VxCamera), _P(VxTraceParams), _vp]),
    ("vx_gen_math", C.c_int, [_vp, C.c_uint32, _vp, C.c_size_t, _vp, _vp]),
    ("vx_gen_math_host", C.c_int, [C.c_uint32, _vp, C.c_size_t, _vp]),
    ("vx_unpack_records", C.c_int,
     [_vp, C.c_size_t, _P(C.c_int32), _P(C.c_uint32), _vp, _vp]),
    ("vx_unpack_compact_records", C.c_int,
     [_vp, C.c_size_t, _P(C.c_int32), _P(C.c_uint32), _vp, _vp]),
    ("vx_render_ao", C.c_int, [_vp, _P(VxCamera), _vp, _vp, _vp]),
    ("vx_render_primary_stats", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams),
                                          _P(C.c_uint64)]),
    ("vx_render_primary_timed", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp, _vp, _vp,
                                          _P(C.c_float)]),
    ("vx_queue_default_tuning", C.c_int, [_P(VxQueueTuning)]),
    ("vx_queue_run", C.c_int, [_vp, _P(C.c_int32), _vp, C.c_size_t, _P(VxTraceParams),
                               _P(VxQueueTuning), _vp, _vp, _vp]),
    ("vx_queue_autotune", C.c_int, [_vp, _P(C.c_int32), _vp, C.c_size_t, _P(VxTraceParams), _vp,
                                    _vp, C.c_int32, _P(VxQueueTuning), _P(C.c_float)]),
    ("vx_queue_graph_create", C.c_int, [_vp, _P(C.c_int32), _vp, C.c_size_t, _P(VxTraceParams),
                                        _P(VxQueueTuning), _vp, _vp, _P(_vp)]),
    ("vx_queue_graph_launch", C.c_int, [_vp, _vp]),
    ("vx_queue_graph_destroy", C.c_int, [_vp]),
    ("vx_server_create", C.c_int, [_vp, _P(C.c_int32), _P(VxTraceParams), _P(VxServeConfig),
                                   _P(_vp)]),
    ("vx_server_submit", C.c_int, [_vp, _vp, C.c_size_t, _vp, _P(C.c_uint64)]),
    ("vx_server_poll", C.c_int, [_vp, C.c_uint64]),
    ("vx_server_wait", C.c_int, [_vp, C.c_uint64, C.c_double]),
    ("vx_server_edit", C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    ("vx_server_stats", C.c_int, [_vp, _P(VxServeStats), C.c_int32]),
    ("vx_server_destroy", C.c_int, [_vp]),
    ("vx_serve_bench", C.c_int, [_vp, _P(VxServeLoad), _P(VxServeStats)]),
    ("vx_project_dirty", C.c_int, [_vp, _P(VxCamera), _vp, C.c_size_t, _vp, _vp]),
    ("vx_tile_refresh", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _vp, _vp]),
    ("vx_render_primary_gated", C.c_int, [_vp, _P(VxCamera), _P(VxTraceParams), _vp, _vp, _vp,
                                          _vp]),
    ("vx_render_primary_noalloc", C.c_int, [_P(VxWorldView), _P(VxCamera), _P(VxTraceParams),
                                            _vp, _vp, _vp]),
    ("vx_wire_query_bytes", C.c_size_t, [C.c_size_t]),
    ("vx_wire_result_bytes", C.c_size_t, [C.c_size_t]),
    ("vx_wire_encode_query", C.c_int, [C.c_uint64, _vp, C.c_size_t, _vp, C.c_size_t,
                                       _P(C.c_size_t)]),
    ("vx_wire_decode_query", C.c_int, [_vp, C.c_size_t, _P(C.c_uint64), _vp, C.c_size_t,
                                       _P(C.c_size_t)]),
    ("vx_wire_encode_result", C.c_int, [C.c_uint64, _vp, C.c_size_t, _vp, C.c_size_t,
                                        _P(C.c_size_t)]),
    ("vx_wire_decode_result", C.c_int, [_vp, C.c_size_t, _P(C.c_uint64), _vp, C.c_size_t,
                                        _P(C.c_size_t)]),
    ("vx_proposal_default_config", C.c_int, [_P(VxTrainConfig)]),
    ("vx_proposal_create", C.c_int, [_vp, C.c_uint64, _P(_vp)]),
    ("vx_proposal_destroy", C.c_int, [_vp]),
    ("vx_proposal_get_params", C.c_int, [_vp, _vp, C.c_size_t]),
    ("vx_proposal_set_params", C.c_int, [_vp, _vp, C.c_size_t]),
    ("vx_proposal_features", C.c_int, [_vp, _vp, _P(C.c_int32), _vp, C.c_size_t, _vp, _vp]),
    ("vx_proposal_grad", C.c_int, [_vp, _vp, _vp, C.c_uint32, _vp, _P(C.c_float)]),
    ("vx_proposal_infer", C.c_int, [_vp, _vp, C.c_size_t, _vp, _vp]),
    ("vx_proposal_train", C.c_int, [_vp, _vp, _P(VxTrainConfig), _vp, _vp]),
    ("vx_render_learned", C.c_int, [_vp, _vp, _P(VxCamera), _P(VxTraceParams), C.c_float, _vp,
                                    _P(VxLearnedStats), _vp]),
    ("vx_host_world_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32, _P(_vp)]),
    ("vx_host_world_destroy", C.c_int, [_vp]),
    ("vx_host_world_arrays", C.c_int, [_vp, _P(_vp), _P(_vp), _P(_vp), _P(_vp), _P(_vp), _P(_vp)]),
    ("vx_host_world_set_voxel", C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint8]),
    ("vx_host_world_apply_edit", C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_uint8,
                                           _P(C.c_int32)]),
    ("vx_host_world_rebuild", C.c_int, [_vp]),
    ("vx_host_world_dirty_count", C.c_int64, [_vp]),
    ("vx_world_sync", C.c_int, [_vp, _vp, _vp]),
]

_lib = None


def load() -> C.CDLL:
    """Load libvoxrt.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH.name} not built at {LIB_PATH}; run python -m voxelg_b200.build")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> int:
    if rc < 0:
        msg = load().vx_last_error()
        raise VxError(rc, msg.decode() if msg else "")
    return rc


def ptr(a) -> int:
    """Address of a numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def i3(v) -> C.Array:
    return (C.c_int32 * 3)(*[int(x) for x in v])


def f3(v) -> C.Array:
    return (C.c_float * 3)(*[float(np.float32(x)) for x in v])
