"""The mixed ray queue: one persistent, graph-captured launch over rays of
any kinds and lengths (vx_queue_* in include/voxrt.h), and the workload
generator of the mixed-queue benchmark."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .world import DeviceWorld


def default_tuning() -> L.VxQueueTuning:
    t = L.VxQueueTuning()
    L.check(L.load().vx_queue_default_tuning(C.byref(t)))
    return t


def _buffers(world: DeviceWorld, rays, out, shadow, with_shadow):
    import torch
    dev = torch.device("cuda", world.device)
    if isinstance(rays, np.ndarray):
        rays = torch.from_numpy(np.ascontiguousarray(rays).view(np.uint8).reshape(-1)).to(dev)
    n = rays.numel() // 32
    if out is None:
        out = torch.empty(n * 24, dtype=torch.uint8, device=dev)
    if shadow is None and with_shadow:
        shadow = torch.empty(n * 8, dtype=torch.uint8, device=dev)
    return rays, n, out, shadow


def run(world: DeviceWorld, rays, params: L.VxTraceParams, tuning=None, origin=(0, 0, 0),
        out=None, shadow=None, with_shadow=True, stream: int = 0):
    """One queue launch; returns (rays, out, shadow) CUDA uint8 tensors."""
    rays, n, out, shadow = _buffers(world, rays, out, shadow, with_shadow)
    L.check(L.load().vx_queue_run(world.handle, L.i3(origin), C.c_void_p(rays.data_ptr()), n,
                                  C.byref(params), C.byref(tuning) if tuning else None,
                                  C.c_void_p(out.data_ptr()),
                                  C.c_void_p(shadow.data_ptr() if shadow is not None else 0),
                                  C.c_void_p(stream)))
    return rays, out, shadow


def autotune(world: DeviceWorld, rays, params: L.VxTraceParams, origin=(0, 0, 0), reps: int = 3,
             out=None, shadow=None, with_shadow=True):
    """Time every candidate tuning (all must give identical records);
    returns (best tuning, best ms, rays, out, shadow)."""
    rays, n, out, shadow = _buffers(world, rays, out, shadow, with_shadow)
    best = L.VxQueueTuning()
    ms = C.c_float()
    L.check(L.load().vx_queue_autotune(world.handle, L.i3(origin), C.c_void_p(rays.data_ptr()), n,
                                       C.byref(params), C.c_void_p(out.data_ptr()),
                                       C.c_void_p(shadow.data_ptr() if shadow is not None else 0),
                                       reps, C.byref(best), C.byref(ms)))
    return best, float(ms.value), rays, out, shadow


class Graph:
    """A queue launch captured in a CUDA graph (fixed buffers)."""

    def __init__(self, world: DeviceWorld, rays, params, tuning=None, origin=(0, 0, 0), out=None,
                 shadow=None, with_shadow=True):
        self.rays, n, self.out, self.shadow = _buffers(world, rays, out, shadow, with_shadow)
        self.n = n
        self._lib = L.load()
        h = C.c_void_p()
        L.check(self._lib.vx_queue_graph_create(
            world.handle, L.i3(origin), C.c_void_p(self.rays.data_ptr()), n, C.byref(params),
            C.byref(tuning) if tuning else None, C.c_void_p(self.out.data_ptr()),
            C.c_void_p(self.shadow.data_ptr() if self.shadow is not None else 0), C.byref(h)))
        self.handle = h

    def launch(self, stream: int = 0):
        L.check(self._lib.vx_queue_graph_launch(self.handle, C.c_void_p(stream)))

    def close(self):
        if getattr(self, "handle", None):
            self._lib.vx_queue_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ workload
def _normalize(v):
    v = v.astype(np.float32)
    n = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])
    return (v / n[:, None]).astype(np.float32)


def primary_dirs(cam: L.VxCamera, width: int, height: int) -> np.ndarray:
    """ray_dir_uv (shaders/raymarch.wgsl:430-438) for every pixel centre."""
    f32 = np.float32
    gx, gy = np.meshgrid(np.arange(width, dtype=np.float32), np.arange(height, dtype=np.float32))
    u = ((gx + f32(0.5)) / f32(cam.res_x)).reshape(-1)
    v = ((gy + f32(0.5)) / f32(cam.res_y)).reshape(-1)
    ndc_x = u * f32(2.0) - f32(1.0)
    ndc_y = f32(1.0) - v * f32(2.0)
    aspect = f32(cam.res_x) / f32(cam.res_y)
    a = ndc_x * f32(cam.tan_half_fov) * aspect
    b = ndc_y * f32(cam.tan_half_fov)
    fw, rt, up = (np.array(list(x), np.float32) for x in (cam.forward, cam.right, cam.up))
    d = (fw[None, :] + rt[None, :] * a[:, None]) + up[None, :] * b[:, None]
    return _normalize(d)


def fibonacci_dirs(n: int = 64) -> np.ndarray:
    """Spherical Fibonacci directions of gi_probes.wgsl:326-330 (one epoch)."""
    k = np.arange(n, dtype=np.float64)
    z = 1.0 - 2.0 * (k + 0.5) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.3999632 * k
    return _normalize(np.stack([r * np.cos(phi), z, r * np.sin(phi)], 1))


def mixed_queue(world_dims, cam: L.VxCamera, width: int, height: int, seed: int,
                probe_radius: int = 256, probe_spacing: int = 16, pick_rays: int = 10000):
    """The mixed-queue workload: every primary ray (flagged to spawn its
    shadow ray), GI-probe rays (64 spherical-Fibonacci directions per probe on
    a 16-voxel grid within 256 voxels of the camera, max length 256) and
    picking rays (max length 8), shuffled with a seeded permutation.
    Returns (rays RAY_DTYPE array, counts dict)."""
    rng = np.random.default_rng(seed)
    vx, vy, vz = world_dims[0] * 4, world_dims[1] * 4, world_dims[2] * 4
    cam_o = np.array(list(cam.origin), np.float32)
    # primaries
    pd = primary_dirs(cam, width, height)
    prim = np.zeros(len(pd), L.RAY_DTYPE)
    prim["org"] = cam_o
    prim["dir"] = pd
    prim["tmax"] = 700.0
    prim["kind"] = L.VX_RAY_SPAWN_SHADOW
    # GI probes: cell centres of the 16-voxel grid in the box of half-size 256
    xs = np.arange(int(cam_o[0]) - probe_radius, int(cam_o[0]) + probe_radius, probe_spacing)
    zs = np.arange(int(cam_o[2]) - probe_radius, int(cam_o[2]) + probe_radius, probe_spacing)
    ys = np.arange(0, vy, probe_spacing)
    xs, zs = xs[(xs >= 0) & (xs < vx)], zs[(zs >= 0) & (zs < vz)]
    sites = np.stack(np.meshgrid(xs, ys, zs, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    sites += np.float32(probe_spacing / 2)
    fd = fibonacci_dirs(64)
    gi = np.zeros(len(sites) * 64, L.RAY_DTYPE)
    gi["org"] = np.repeat(sites, 64, axis=0)
    gi["dir"] = np.tile(fd, (len(sites), 1))
    gi["tmax"] = 256.0
    gi["kind"] = 0
    # picking rays: random origins in the window, random directions, length 8
    pk = np.zeros(pick_rays, L.RAY_DTYPE)
    pk["org"] = rng.uniform([0, 0, 0], [vx, vy, vz], size=(pick_rays, 3)).astype(np.float32)
    pk["dir"] = _normalize(rng.normal(size=(pick_rays, 3)))
    pk["tmax"] = 8.0
    pk["kind"] = 0
    rays = np.concatenate([prim, gi, pk])
    rays = rays[rng.permutation(len(rays))]
    return rays, {"primary": len(prim), "gi_probe": len(gi), "picking": len(pk),
                  "probes": len(sites)}
