"""Traversal entry points over a DeviceWorld.

* ``raycast`` mirrors voxelG's picking call
  ``raycast(camera_world, dir, world, world_origin) -> Option<PickHit>``
  (src/raycast.rs:21).
* ``render_primary`` runs one primary frame: beam pre-pass, per-pixel
  hierarchical trace and one shadow ray per hit (shaders/beam.wgsl:30-113,
  shaders/raymarch.wgsl:576-631, :3953-3994).
* ``trace`` runs a batch of generic rays (trace / trace_any / trace_no_water).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib as L
from .world import DeviceWorld

KIND_TRACE = 0
KIND_ANY = 1
KIND_NO_WATER = 2


@dataclass
class PickHit:
    """src/raycast.rs:13-17"""
    voxel: tuple
    normal: tuple


def default_params(flags: Optional[int] = None, frame: float = 0.0) -> L.VxTraceParams:
    p = L.VxTraceParams()
    L.check(L.load().vx_default_params(C.byref(p)))
    if flags is not None:
        p.flags = flags
    p.frame = frame
    return p


def camera_from_pose(pos, yaw: float, pitch: float, fov_y: float, width: int, height: int,
                     world_origin=(0, 0, 0)) -> L.VxCamera:
    """CameraUniform::from_camera (src/camera.rs:25-42, :140-166)."""
    cam = L.VxCamera()
    L.check(L.load().vx_camera_from_pose(L.f3(pos), yaw, pitch, fov_y, width, height,
                                         L.i3(world_origin), C.byref(cam)))
    return cam


def default_camera(world: DeviceWorld | tuple, width: int, height: int) -> L.VxCamera:
    """The workloads' camera: window centre at y=140, pitch -15 deg, yaw 0,
    vfov 70 deg."""
    dims = world.dims if isinstance(world, DeviceWorld) else world
    cx, cz = dims[0] * 4 // 2, dims[2] * 4 // 2
    return camera_from_pose((cx, 140.0, cz), 0.0, math.radians(-15.0), math.radians(70.0),
                            width, height)


def raycast(camera_world, dir, world: DeviceWorld, world_origin=(0, 0, 0)) -> Optional[PickHit]:
    """Drop-in for voxelG's raycast(): first solid non-fringe voxel along the
    ray and its entry normal, or None (miss, zero direction, step cap)."""
    out = L.VxPickHit()
    rc = L.check(L.load().vx_raycast(world.handle, L.f3(camera_world), L.f3(dir),
                                     L.i3(world_origin), C.byref(out)))
    if rc == 0:
        return None
    return PickHit(tuple(out.voxel), tuple(out.normal))


def _torch():
    import torch
    return torch


def render_primary(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams, rec=None,
                   shadow=None, stream: int = 0):
    """Device-side frame.  rec/shadow are uint8 CUDA tensors (allocated when
    None); returns (rec, shadow)."""
    torch = _torch()
    n = int(cam.res_x) * int(cam.res_y)
    dev = torch.device("cuda", world.device)
    if rec is None:
        rec = torch.empty(n * 24, dtype=torch.uint8, device=dev)
    if shadow is None and (params.flags & L.VX_F_SHADOW):
        shadow = torch.empty(n * 8, dtype=torch.uint8, device=dev)
    L.check(L.load().vx_render_primary(world.handle, C.byref(cam), C.byref(params),
                                       C.c_void_p(rec.data_ptr()),
                                       C.c_void_p(shadow.data_ptr() if shadow is not None else 0),
                                       C.c_void_p(stream)))
    return rec, shadow


def render_primary_rows(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams, y0: int,
                        y1: int, rec, shadow=None, stream: int = 0):
    """Rows [y0, y1) of the frame into rec / shadow (uint8 CUDA tensors of at
    least y1 * res_x records), at their frame positions; other rows are left
    as they were."""
    n = int(y1) * int(cam.res_x)
    if rec.numel() < n * 24 or (shadow is not None and shadow.numel() < n * 8):
        raise ValueError("render_primary_rows: buffers hold fewer than y1 * res_x records")
    L.check(L.load().vx_render_primary_rows(world.handle, C.byref(cam), C.byref(params),
                                            int(y0), int(y1), C.c_void_p(rec.data_ptr()),
                                            C.c_void_p(shadow.data_ptr() if shadow is not None else 0),
                                            C.c_void_p(stream)))
    return rec, shadow


def tile_mask_words(width: int, height: int) -> int:
    """u32 words of an 8x8-tile dirty mask (src/app.rs:643-648)."""
    return ((width + 7) // 8 * ((height + 7) // 8) + 31) // 32


def project_dirty(world: DeviceWorld, cam: L.VxCamera, brick_idx, mask, stream: int = 0):
    """OR the screen tiles covered by the given slot bricks into mask (a CUDA
    int32 tensor of tile_mask_words entries), temporal.rs:16-111."""
    idx = np.ascontiguousarray(brick_idx, dtype=np.uint32)
    L.check(L.load().vx_project_dirty(world.handle, C.byref(cam), C.c_void_p(L.ptr(idx)),
                                      len(idx), C.c_void_p(mask.data_ptr()), C.c_void_p(stream)))
    return mask


def tile_refresh(width: int, height: int, spread: int, phase: int, mask, stream: int = 0):
    """OR the rotating refresh set of src/app.rs:706-725 into mask."""
    L.check(L.load().vx_tile_refresh(width, height, spread, phase, C.c_void_p(mask.data_ptr()),
                                     C.c_void_p(stream)))
    return mask


def render_primary_gated(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams, mask,
                         rec, shadow=None, stream: int = 0):
    """Frame with cs_main's tile gate: only dirty tiles are re-traced into
    rec/shadow (CUDA uint8 tensors holding the previous frame)."""
    L.check(L.load().vx_render_primary_gated(
        world.handle, C.byref(cam), C.byref(params), C.c_void_p(mask.data_ptr()),
        C.c_void_p(rec.data_ptr()), C.c_void_p(shadow.data_ptr() if shadow is not None else 0),
        C.c_void_p(stream)))
    return rec, shadow


def render_primary_host(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams,
                        rec_host: Optional[np.ndarray] = None,
                        shadow_host: Optional[np.ndarray] = None):
    """Frame through host buffers (copies included); returns numpy records."""
    n = int(cam.res_x) * int(cam.res_y)
    if rec_host is None:
        rec_host = np.empty(n, L.RECORD_DTYPE)
    if shadow_host is None and (params.flags & L.VX_F_SHADOW):
        shadow_host = np.empty(n, L.SHADOW_DTYPE)
    L.check(L.load().vx_render_primary_host(
        world.handle, C.byref(cam), C.byref(params), C.c_void_p(L.ptr(rec_host)),
        C.c_void_p(L.ptr(shadow_host) if shadow_host is not None else 0)))
    return rec_host, shadow_host


def render_primary_host_async(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams,
                              rec_host: np.ndarray, shadow_host: Optional[np.ndarray] = None):
    """Enqueue a frame into host buffers (pinned) and return at once; the
    records are there after render_host_wait(world).  Successive frames
    overlap: one renders while the previous one copies."""
    L.check(L.load().vx_render_primary_host_async(
        world.handle, C.byref(cam), C.byref(params), C.c_void_p(L.ptr(rec_host)),
        C.c_void_p(L.ptr(shadow_host) if shadow_host is not None else 0)))


def render_primary_host_packed(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams,
                               out: Optional[np.ndarray] = None) -> np.ndarray:
    """Frame through a host buffer of 16-byte packed records (records and
    shadow records, losslessly); returns the PACKED_DTYPE array."""
    n = int(cam.res_x) * int(cam.res_y)
    if out is None:
        out = np.empty(n, L.PACKED_DTYPE)
    L.check(L.load().vx_render_primary_host_packed(world.handle, C.byref(cam), C.byref(params),
                                                   C.c_void_p(L.ptr(out))))
    return out


def render_primary_host_packed_async(world: DeviceWorld, cam: L.VxCamera,
                                     params: L.VxTraceParams, out: np.ndarray):
    """Enqueue a packed frame into a (pinned) host buffer; it is there after
    render_host_wait(world)."""
    L.check(L.load().vx_render_primary_host_packed_async(world.handle, C.byref(cam),
                                                         C.byref(params), C.c_void_p(L.ptr(out))))


def unpack_records(packed: np.ndarray, world_origin, window_voxels):
    """Packed records back to (RECORD_DTYPE, SHADOW_DTYPE) arrays."""
    packed = np.ascontiguousarray(packed).view(L.PACKED_DTYPE)
    n = len(packed)
    rec = np.empty(n, L.RECORD_DTYPE)
    sh = np.empty(n, L.SHADOW_DTYPE)
    wv = (C.c_uint32 * 3)(*[int(v) for v in window_voxels])
    L.check(L.load().vx_unpack_records(C.c_void_p(L.ptr(packed)), n, L.i3(world_origin), wv,
                                       C.c_void_p(L.ptr(rec)), C.c_void_p(L.ptr(sh))))
    return rec, sh


def render_primary_host_compact(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams,
                                out: Optional[np.ndarray] = None) -> np.ndarray:
    """Frame through a host buffer of 12-byte compact records (records and
    shadow records, losslessly); returns the COMPACT_DTYPE array."""
    n = int(cam.res_x) * int(cam.res_y)
    if out is None:
        out = np.empty(n, L.COMPACT_DTYPE)
    L.check(L.load().vx_render_primary_host_compact(world.handle, C.byref(cam), C.byref(params),
                                                    C.c_void_p(L.ptr(out))))
    return out


def render_primary_host_compact_async(world: DeviceWorld, cam: L.VxCamera,
                                      params: L.VxTraceParams, out: np.ndarray):
    """Enqueue a compact frame into a (pinned) host buffer; it is there after
    render_host_wait(world)."""
    L.check(L.load().vx_render_primary_host_compact_async(world.handle, C.byref(cam),
                                                          C.byref(params), C.c_void_p(L.ptr(out))))


def unpack_compact_records(compact: np.ndarray, world_origin, window_voxels):
    """Compact records back to (RECORD_DTYPE, SHADOW_DTYPE) arrays."""
    compact = np.ascontiguousarray(compact).view(L.COMPACT_DTYPE)
    n = len(compact)
    rec = np.empty(n, L.RECORD_DTYPE)
    sh = np.empty(n, L.SHADOW_DTYPE)
    wv = (C.c_uint32 * 3)(*[int(v) for v in window_voxels])
    L.check(L.load().vx_unpack_compact_records(C.c_void_p(L.ptr(compact)), n,
                                               L.i3(world_origin), wv, C.c_void_p(L.ptr(rec)),
                                               C.c_void_p(L.ptr(sh))))
    return rec, sh


def render_host_wait(world: DeviceWorld):
    """Wait until every enqueued host-buffer frame has landed."""
    L.check(L.load().vx_render_host_wait(world.handle))


def render_ao(world: DeviceWorld, cam: L.VxCamera, rec, ao=None, stream: int = 0):
    """Contact AO of a frame's primary records (rec: CUDA uint8 tensor from
    render_primary with the same camera); returns a float32 CUDA tensor."""
    torch = _torch()
    n = int(cam.res_x) * int(cam.res_y)
    if ao is None:
        ao = torch.empty(n, dtype=torch.float32, device=rec.device)
    L.check(L.load().vx_render_ao(world.handle, C.byref(cam), C.c_void_p(rec.data_ptr()),
                                  C.c_void_p(ao.data_ptr()), C.c_void_p(stream)))
    return ao


def render_stats(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams):
    """Algorithmic bytes and loop iterations of one frame:
    {"beam": (bytes, iters), "primary": (bytes, iters)} (primary includes
    the shadow rays)."""
    s = (C.c_uint64 * 4)()
    L.check(L.load().vx_render_primary_stats(world.handle, C.byref(cam), C.byref(params), s))
    return {"beam": (int(s[0]), int(s[1])), "primary": (int(s[2]), int(s[3]))}


def render_primary_timed(world: DeviceWorld, cam: L.VxCamera, params: L.VxTraceParams, rec,
                         shadow=None, stream: int = 0):
    """One device frame with CUDA events around each kernel on `stream`;
    returns (beam_ms, primary_ms).  Synchronizes."""
    ms = (C.c_float * 2)()
    L.check(L.load().vx_render_primary_timed(
        world.handle, C.byref(cam), C.byref(params), C.c_void_p(rec.data_ptr()),
        C.c_void_p(shadow.data_ptr() if shadow is not None else 0), C.c_void_p(stream), ms))
    return float(ms[0]), float(ms[1])


def trace(world: DeviceWorld, rays, params: L.VxTraceParams, origin=(0, 0, 0), out=None,
          stream: int = 0):
    """Batched generic rays.  rays: CUDA uint8 tensor of n*32 bytes (RAY_DTYPE
    rows) or a numpy RAY_DTYPE array (copied to the device).  Returns a CUDA
    uint8 tensor of n*24 record bytes."""
    torch = _torch()
    dev = torch.device("cuda", world.device)
    if isinstance(rays, np.ndarray):
        rays = torch.from_numpy(np.ascontiguousarray(rays).view(np.uint8).reshape(-1)).to(dev)
    n = rays.numel() // 32
    if out is None:
        out = torch.empty(n * 24, dtype=torch.uint8, device=dev)
    L.check(L.load().vx_trace(world.handle, L.i3(origin), C.c_void_p(rays.data_ptr()), n,
                              C.byref(params), C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out


def raycast_batch(world: DeviceWorld, cams: np.ndarray, dirs: np.ndarray, origin=(0, 0, 0)):
    """Batched picking on the device; returns (hits PICK_DTYPE, hit flags)."""
    torch = _torch()
    dev = torch.device("cuda", world.device)
    n = len(cams)
    c = torch.from_numpy(np.ascontiguousarray(cams, dtype=np.float32).reshape(-1)).to(dev)
    d = torch.from_numpy(np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1)).to(dev)
    out = torch.empty(n * 24, dtype=torch.uint8, device=dev)
    hit = torch.empty(n, dtype=torch.int32, device=dev)
    L.check(L.load().vx_raycast_batch(world.handle, L.i3(origin), C.c_void_p(c.data_ptr()),
                                      C.c_void_p(d.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                      C.c_void_p(hit.data_ptr()), C.c_void_p(0)))
    torch.cuda.synchronize(dev)
    return out.cpu().numpy().view(L.PICK_DTYPE), hit.cpu().numpy()


def records(t) -> np.ndarray:
    """uint8 tensor/array -> RECORD_DTYPE numpy view."""
    a = t.cpu().numpy() if hasattr(t, "cpu") else t
    return np.ascontiguousarray(a).view(L.RECORD_DTYPE)


def shadows(t) -> np.ndarray:
    a = t.cpu().numpy() if hasattr(t, "cpu") else t
    return np.ascontiguousarray(a).view(L.SHADOW_DTYPE)
