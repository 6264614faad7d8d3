"""ctypes binding of the CPU oracle (voxoracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product (libvoxrt) never
uses it.  Struct layouts are defined here independently of the product's
binding; they are byte-identical by construction of the record contract.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "libvoxoracle.so"

OR_F_L4, OR_F_LUT, OR_F_LOD, OR_F_BEAM, OR_F_SHADOW = 1, 2, 4, 8, 16

BRICK = np.dtype([("occupancy", "<u8"), ("materials", "u1", (64,))])
RECORD = np.dtype([("voxel", "<i4", (3,)), ("face", "u1"), ("mat", "u1"), ("flags", "u1"),
                   ("pad", "u1"), ("t", "<f4"), ("steps", "<u4")])
SHADOW = np.dtype([("steps", "<u4"), ("occluded", "u1"), ("traced", "u1"), ("pad", "<u2")])
RAY = np.dtype([("org", "<f4", (3,)), ("dir", "<f4", (3,)), ("tmax", "<f4"), ("kind", "<u4")])
PICK = np.dtype([("voxel", "<i4", (3,)), ("normal", "<i4", (3,))])


class OrWorld(C.Structure):
    _fields_ = [("bx", C.c_int32), ("by", C.c_int32), ("bz", C.c_int32),
                ("bricks", C.c_void_p), ("tile_mask", C.c_void_p), ("chunk_mask", C.c_void_p),
                ("l4_mask", C.c_void_p), ("brick_uniform", C.c_void_p),
                ("tile_uniform", C.c_void_p)]


class OrCamera(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("tan_half_fov", C.c_float), ("res_x", C.c_float),
                ("res_y", C.c_float), ("jitter_x", C.c_float), ("jitter_y", C.c_float),
                ("world_origin", C.c_int32 * 3)]


class OrParams(C.Structure):
    _fields_ = [("max_dist", C.c_float), ("lod_brick_t", C.c_float), ("tile_lod_t", C.c_float),
                ("shadow_max_dist", C.c_float), ("beam_margin", C.c_float),
                ("max_iters", C.c_int32), ("any_max_iters", C.c_int32), ("flags", C.c_uint32),
                ("sun", C.c_float * 3), ("sun_tangent", C.c_float * 3),
                ("sun_bitangent", C.c_float * 3), ("cone_tan", C.c_float), ("frame", C.c_float)]


class OrTerrain(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("base_height", C.c_float), ("amplitude", C.c_float),
                ("inv_wavelength", C.c_float), ("octaves", C.c_uint32),
                ("water_level", C.c_int32), ("cave_inv_wavelength", C.c_float),
                ("cave_threshold", C.c_float), ("dirt_depth", C.c_int32)]


class OrPickHit(C.Structure):
    _fields_ = [("voxel", C.c_int32 * 3), ("normal", C.c_int32 * 3)]


class OrStats(C.Structure):
    _fields_ = [("bytes", C.c_uint64), ("iters", C.c_uint64)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "or_libm_batch": (None, [C.c_int, vp, C.c_size_t, vp, C.c_int]),
        "or_rebuild_all_masks": (None, [P(OrWorld)]),
        "or_rebuild_all_uniform": (None, [P(OrWorld)]),
        "or_set_voxel": (C.c_int64, [P(OrWorld), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint8]),
        "or_generate_terrain": (None, [P(OrWorld), P(OrTerrain), C.c_int]),
        "or_sample_terrain": (C.c_int32, [C.c_float, C.c_float, C.c_uint64, P(C.c_int32)]),
        "or_trees_for_chunk": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, vp]),
        "or_gen_slot_bricks": (None, [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, vp]),
        "or_fill_window": (None, [P(OrWorld), C.c_uint64, C.c_int32, C.c_int32, C.c_int]),
        "or_fbm_2d": (C.c_float, [C.c_float, C.c_float, C.c_uint32]),
        "or_value_noise_3d": (C.c_float, [C.c_float, C.c_float, C.c_float]),
        "or_ray_dir_uv": (None, [P(OrCamera), C.c_float, C.c_float, P(C.c_float)]),
        "or_sincos": (None, [C.c_float, P(C.c_float), P(C.c_float)]),
        "or_ign": (C.c_float, [C.c_float, C.c_float, C.c_float]),
        "or_raycast": (C.c_int, [P(OrWorld), P(C.c_float), P(C.c_float), P(C.c_int32),
                                 P(OrPickHit), P(C.c_uint32)]),
        "or_trace": (None, [P(OrWorld), P(C.c_int32), P(C.c_float), P(C.c_float), C.c_float,
                            P(OrParams), vp, P(OrStats)]),
        "or_trace_any": (C.c_int, [P(OrWorld), P(C.c_int32), P(C.c_float), P(C.c_float),
                                   C.c_float, P(OrParams), P(C.c_uint32), P(OrStats)]),
        "or_beam_pass": (None, [P(OrWorld), P(OrCamera), vp, P(OrStats)]),
        "or_render_frame": (C.c_double, [P(OrWorld), P(OrCamera), P(OrParams), vp, vp, vp,
                                         C.c_int, P(OrStats)]),
        "or_render_rows": (None, [P(OrWorld), P(OrCamera), P(OrParams), vp, C.c_uint32,
                                  C.c_uint32, vp, vp, P(OrStats)]),
        "or_project_brick_to_tiles": (None, [P(OrWorld), P(OrCamera), C.c_uint32, vp]),
        "or_compute_ao": (C.c_float, [P(OrWorld), P(OrCamera), vp, C.c_uint32, C.c_uint32]),
        "or_render_ao": (None, [P(OrWorld), P(OrCamera), vp, vp, C.c_int]),
        "or_refresh_tiles": (None, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp]),
        "or_render_row_set": (C.c_double, [P(OrWorld), P(OrCamera), P(OrParams), vp, C.c_uint32,
                                           C.c_uint32, vp, vp, C.c_int, P(OrStats)]),
        "or_trace_batch": (C.c_double, [P(OrWorld), P(C.c_int32), vp, C.c_size_t, P(OrParams),
                                        vp, vp, C.c_int, P(OrStats)]),
        "or_raycast_batch": (C.c_double, [P(OrWorld), P(C.c_int32), vp, vp, C.c_size_t, vp, vp,
                                          C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def counts(bx, by, bz):
    tx, ty, tz = bx // 4, by // 4, bz // 4
    cx, cy, cz = (tx + 3) // 4, (ty + 3) // 4, (tz + 3) // 4
    lx, ly, lz = (cx + 3) // 4, (cy + 3) // 4, (cz + 3) // 4
    return bx * by * bz, tx * ty * tz, cx * cy * cz, lx * ly * lz


class World:
    """Oracle-side world: numpy arrays in voxelG's host layout."""

    NAMES = ("bricks", "tile_mask", "chunk_mask", "l4_mask", "brick_uniform", "tile_uniform")

    def __init__(self, bx, by, bz, arrays=None):
        self.dims = (bx, by, bz)
        nb, nt, nc, nl = counts(bx, by, bz)
        if arrays is None:
            arrays = {"bricks": np.zeros(nb, BRICK), "tile_mask": np.zeros(nt, np.uint64),
                      "chunk_mask": np.zeros(nc, np.uint64), "l4_mask": np.zeros(nl, np.uint64),
                      "brick_uniform": np.zeros(nb, np.uint8),
                      "tile_uniform": np.zeros(nt, np.uint8)}
        self.a = {k: np.ascontiguousarray(arrays[k]) for k in self.NAMES}
        self.a["bricks"] = self.a["bricks"].view(BRICK)
        self.c = OrWorld(bx, by, bz, *[self.a[k].ctypes.data for k in self.NAMES])

    @property
    def voxels(self):
        return (self.dims[0] * 4, self.dims[1] * 4, self.dims[2] * 4)

    def rebuild(self):
        load().or_rebuild_all_masks(C.byref(self.c))
        load().or_rebuild_all_uniform(C.byref(self.c))

    def set_voxel(self, x, y, z, m):
        return load().or_set_voxel(C.byref(self.c), x, y, z, m)

    def generate(self, terrain, threads=None):
        t = OrTerrain(terrain.seed, terrain.base_height, terrain.amplitude,
                      terrain.inv_wavelength, terrain.octaves, terrain.water_level,
                      terrain.cave_inv_wavelength, terrain.cave_threshold, terrain.dirt_depth)
        load().or_generate_terrain(C.byref(self.c), C.byref(t), threads or os.cpu_count() or 1)
        self.rebuild()


TREE = np.dtype([("base", "<i4", 3), ("ttype", "<u4"), ("hash", "<u4")])


def gen_slot_bricks(cx, cy, cz, seed):
    """The reference's chunk generator for world chunk (cx, cy, cz): 512
    bricks in scratch order x + y*8 + z*64 (voxel.rs:1322-1500)."""
    out = np.zeros(512, BRICK)
    load().or_gen_slot_bricks(cx, cy, cz, C.c_uint64(seed & (2**64 - 1)), out.ctypes.data)
    return out


def sample_terrain(wx, wz, seed):
    """(height, water_top) of one column (voxel.rs:1244-1316)."""
    wt = C.c_int32()
    h = load().or_sample_terrain(float(np.float32(wx)), float(np.float32(wz)),
                                 C.c_uint64(seed & (2**64 - 1)), C.byref(wt))
    return h, wt.value


def trees_for_chunk(cx, cz, seed):
    out = np.zeros(12, TREE)
    n = load().or_trees_for_chunk(cx, cz, C.c_uint64(seed & (2**64 - 1)), out.ctypes.data)
    return out[:n]


def fill_window(world: "World", seed, ox=0, oz=0, threads=None):
    """fill_demo_terrain for a window whose lower corner is world chunk
    (ox, 0, oz): every slot generated by gen_slot_bricks, masks rebuilt."""
    load().or_fill_window(C.byref(world.c), C.c_uint64(seed & (2**64 - 1)), ox, oz,
                          threads or os.cpu_count() or 1)


def params_from(p) -> OrParams:
    """Copy a product VxTraceParams (or any object with the same fields)."""
    q = OrParams()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(OrParams))
    return q


def camera_from(c) -> OrCamera:
    q = OrCamera()
    C.memmove(C.byref(q), C.byref(c), C.sizeof(OrCamera))
    return q


def f3(v):
    return (C.c_float * 3)(*[float(np.float32(x)) for x in v])


def i3(v):
    return (C.c_int32 * 3)(*[int(x) for x in v])


def render_frame(world: World, cam, params, threads=None, stats=False):
    """Full frame: (records, shadows, beam, seconds, OrStats)."""
    cam = camera_from(cam)
    p = params_from(params)
    W, H = int(cam.res_x), int(cam.res_y)
    rec = np.zeros(W * H, RECORD)
    sh = np.zeros(W * H, SHADOW)
    beam = np.zeros(((W + 7) // 8) * ((H + 7) // 8), np.float32)
    st = OrStats()
    secs = load().or_render_frame(C.byref(world.c), C.byref(cam), C.byref(p), rec.ctypes.data,
                                  sh.ctypes.data, beam.ctypes.data, threads or os.cpu_count() or 1,
                                  C.byref(st))
    return rec, sh, beam, secs, st


def render_rows(world: World, cam, params, beam, y0, y1):
    """Rows [y0, y1) of a frame given a beam buffer (single thread)."""
    cam = camera_from(cam)
    p = params_from(params)
    W = int(cam.res_x)
    rec = np.zeros(W * int(cam.res_y), RECORD)
    sh = np.zeros(W * int(cam.res_y), SHADOW)
    st = OrStats()
    load().or_render_rows(C.byref(world.c), C.byref(cam), C.byref(p), beam.ctypes.data, y0, y1,
                          rec.ctypes.data, sh.ctypes.data, C.byref(st))
    return rec[y0 * W:y1 * W], sh[y0 * W:y1 * W], st


def render_row_set(world: World, cam, params, beam, stride, offset, threads=None):
    """Rows offset, offset+stride, ... of a frame on all threads: (records of
    those rows, shadows of those rows, seconds, OrStats)."""
    cam = camera_from(cam)
    p = params_from(params)
    W, H = int(cam.res_x), int(cam.res_y)
    rec = np.zeros(W * H, RECORD)
    sh = np.zeros(W * H, SHADOW)
    st = OrStats()
    secs = load().or_render_row_set(C.byref(world.c), C.byref(cam), C.byref(p),
                                    beam.ctypes.data, stride, offset, rec.ctypes.data,
                                    sh.ctypes.data, threads or os.cpu_count() or 1, C.byref(st))
    rows = np.arange(offset, H, stride)
    idx = (rows[:, None] * W + np.arange(W)[None, :]).reshape(-1)
    return rec[idx], sh[idx], secs, st


def render_ao(world: World, cam, rec: np.ndarray, threads=None) -> np.ndarray:
    """Contact AO (compute_ao, raymarch.wgsl:4417-4453) of every primary
    record of a frame of `cam`; 1.0 for misses and skipped hits."""
    cam = camera_from(cam)
    rec = np.ascontiguousarray(rec).view(RECORD)
    ao = np.empty(len(rec), np.float32)
    load().or_render_ao(C.byref(world.c), C.byref(cam), rec.ctypes.data, ao.ctypes.data,
                        threads or os.cpu_count() or 1)
    return ao


def project_dirty(world: World, cam, brick_idx, mask=None):
    """temporal.rs:16-111 over a list of slot bricks -> u32 tile mask."""
    cam = camera_from(cam)
    W, H = int(cam.res_x), int(cam.res_y)
    if mask is None:
        mask = np.zeros((((W + 7) // 8) * ((H + 7) // 8) + 31) // 32, np.uint32)
    for bi in brick_idx:
        load().or_project_brick_to_tiles(C.byref(world.c), C.byref(cam), int(bi), mask.ctypes.data)
    return mask


def refresh_tiles(W, H, spread, phase, mask):
    load().or_refresh_tiles((W + 7) // 8, (H + 7) // 8, spread, phase, mask.ctypes.data)
    return mask


def beam_pass(world: World, cam):
    cam = camera_from(cam)
    W, H = int(cam.res_x), int(cam.res_y)
    beam = np.zeros(((W + 7) // 8) * ((H + 7) // 8), np.float32)
    st = OrStats()
    load().or_beam_pass(C.byref(world.c), C.byref(cam), beam.ctypes.data, C.byref(st))
    return beam, st


def trace_batch(world: World, rays: np.ndarray, params, origin=(0, 0, 0), threads=None,
                shadows=False):
    """The mixed queue on the CPU: (records, seconds, OrStats) or, with
    shadows=True, (records, shadow records, seconds, OrStats)."""
    p = params_from(params)
    rays = np.ascontiguousarray(rays).view(RAY)
    out = np.zeros(len(rays), RECORD)
    sh = np.zeros(len(rays), SHADOW) if shadows else None
    st = OrStats()
    secs = load().or_trace_batch(C.byref(world.c), i3(origin), rays.ctypes.data, len(rays),
                                 C.byref(p), out.ctypes.data, sh.ctypes.data if shadows else None,
                                 threads or os.cpu_count() or 1, C.byref(st))
    if shadows:
        return out, sh, secs, st
    return out, secs, st


def raycast(world: World, cam, d, origin=(0, 0, 0)):
    """O1 (src/raycast.rs): (hit, voxel, normal, steps)."""
    out = OrPickHit()
    steps = C.c_uint32()
    hit = load().or_raycast(C.byref(world.c), f3(cam), f3(d), i3(origin), C.byref(out),
                            C.byref(steps))
    return bool(hit), tuple(out.voxel), tuple(out.normal), int(steps.value)


def raycast_batch(world: World, cams, dirs, origin=(0, 0, 0), threads=None):
    cams = np.ascontiguousarray(cams, dtype=np.float32)
    dirs = np.ascontiguousarray(dirs, dtype=np.float32)
    n = len(cams)
    out = np.zeros(n, PICK)
    hit = np.zeros(n, np.int32)
    secs = load().or_raycast_batch(C.byref(world.c), i3(origin), cams.ctypes.data,
                                   dirs.ctypes.data, n, out.ctypes.data, hit.ctypes.data,
                                   threads or os.cpu_count() or 1)
    return out, hit, secs


def trace_one(world: World, origin_world, d, params, ro=(0, 0, 0), max_dist=None):
    p = params_from(params)
    rec = np.zeros(1, RECORD)
    st = OrStats()
    load().or_trace(C.byref(world.c), i3(ro), f3(origin_world), f3(d),
                    float(p.max_dist if max_dist is None else max_dist), C.byref(p),
                    rec.ctypes.data, C.byref(st))
    return rec[0], st


def trace_any_one(world: World, origin_world, d, params, ro=(0, 0, 0), max_dist=None):
    p = params_from(params)
    steps = C.c_uint32()
    st = OrStats()
    occ = load().or_trace_any(C.byref(world.c), i3(ro), f3(origin_world), f3(d),
                              float(p.shadow_max_dist if max_dist is None else max_dist),
                              C.byref(p), C.byref(steps), C.byref(st))
    return bool(occ), int(steps.value)


def ray_dir_uv(cam, u: float, v: float):
    """ray_dir_uv (raymarch.wgsl:430-438) of a camera at screen (u, v)."""
    out = (C.c_float * 3)()
    load().or_ray_dir_uv(C.byref(camera_from(cam)), u, v, out)
    return tuple(out)


def camera_from_pose(pos, yaw, pitch, fov_y, width, height, world_origin=(0, 0, 0)) -> OrCamera:
    """src/camera.rs:25-42 (basis) and :140-166 (uniform) in f32 numpy."""
    import math
    f = np.float32

    def norm(v):
        v = np.asarray(v, np.float32)
        r = f(1.0) / np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
        return np.array([v[0] * r, v[1] * r, v[2] * r], np.float32)

    fw = norm([f(math.sin(f(yaw))) * f(math.cos(f(pitch))), f(math.sin(f(pitch))),
               f(math.cos(f(yaw))) * f(math.cos(f(pitch)))])
    rt = norm([fw[2], f(0.0), -fw[0]])
    up = norm([fw[1] * rt[2] - rt[1] * fw[2], fw[2] * rt[0] - rt[2] * fw[0],
               fw[0] * rt[1] - rt[0] * fw[1]])
    c = OrCamera()
    for k in range(3):
        c.origin[k], c.forward[k], c.right[k], c.up[k] = float(pos[k]), fw[k], rt[k], up[k]
        c.world_origin[k] = int(world_origin[k])
    c.tan_half_fov = float(f(math.tan(f(f(fov_y) * f(0.5)))))
    c.res_x, c.res_y = float(width), float(height)
    return c


def default_params(flags=OR_F_L4 | OR_F_LUT | OR_F_LOD | OR_F_BEAM | OR_F_SHADOW,
                   frame=0.0) -> OrParams:
    """Reference constants (raymarch.wgsl:4489-4526, :4625, :4359, :608) and
    the workload's sun: normalize(0.3, 0.8, 0.5), tangent frame as
    raymarch.wgsl:3984-3988, tan(0.5 deg) cone."""
    f = np.float32
    p = OrParams()
    p.max_dist, p.lod_brick_t, p.tile_lod_t = 700.0, 400.0, 520.0
    p.shadow_max_dist, p.beam_margin = 480.0, 16.0
    p.max_iters, p.any_max_iters, p.flags = 1024, 768, flags
    s = np.array([0.3, 0.8, 0.5], np.float32)
    sl = np.sqrt((s[0] * s[0] + s[1] * s[1]) + s[2] * s[2])
    s = np.array([s[0] / sl, s[1] / sl, s[2] / sl], np.float32)
    t = np.array([-s[2], f(0.0), s[0]], np.float32)
    tl = np.sqrt((t[0] * t[0] + t[1] * t[1]) + t[2] * t[2])
    if tl < f(0.01):
        t = np.array([1.0, 0.0, 0.0], np.float32)
    else:
        t = np.array([t[0] / tl, t[1] / tl, t[2] / tl], np.float32)
    b = np.array([s[1] * t[2] - s[2] * t[1], s[2] * t[0] - s[0] * t[2],
                  s[0] * t[1] - s[1] * t[0]], np.float32)
    for k in range(3):
        p.sun[k], p.sun_tangent[k], p.sun_bitangent[k] = float(s[k]), float(t[k]), float(b[k])
    p.cone_tan = float(f(0.0087268678))
    p.frame = float(f(frame))
    return p


def libm_batch(fn: int, x: np.ndarray, threads=None) -> np.ndarray:
    """glibc powf(x, 1.15f) (fn 0), powf(x, 0.85f) (1), cosf (2), sinf (3)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    load().or_libm_batch(fn, x.ctypes.data, len(x), out.ctypes.data, threads or os.cpu_count() or 1)
    return out
