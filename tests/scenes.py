"""Crafted test worlds and ray fans restated from the reference's own parity
tests (src/accel.rs:505-942), built on the oracle's world arrays.

Each builder returns an oracle World with voxelG's default dims
(128 x 64 x 128 bricks = 512 x 256 x 512 voxels, src/world_dims.rs:12-14).
"""
from __future__ import annotations

import numpy as np

from oracle import pyoracle as po

DEFAULT_BRICKS = (128, 64, 128)
MAT_STONE = 4
f32 = np.float32


def normalize(v):
    """glam Vec3::normalize: v * (1 / sqrt(dot(v, v))) in f32."""
    v = np.asarray(v, np.float32)
    r = f32(1.0) / np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return np.array([v[0] * r, v[1] * r, v[2] * r], np.float32)


def apply_edit(w: po.World, wx, wy, wz, mat, origin):
    """World::apply_edit, src/voxel.rs:450-474 (toroidal slot mapping)."""
    vx, vy, vz = w.voxels
    rx, ry, rz = wx - origin[0], wy - origin[1], wz - origin[2]
    if rx < 0 or ry < 0 or rz < 0 or rx >= vx or ry >= vy or rz >= vz:
        return
    w.set_voxel(wx % vx, ry, wz % vz, mat)


def flat_floor(x0, z0, n) -> po.World:
    """accel.rs:505-527: stone floor, top solid layer y=60, x,z in [x0, x0+n)."""
    w = po.World(*DEFAULT_BRICKS)
    for z in range(z0, z0 + n):
        for x in range(x0, x0 + n):
            for y in range(57, 61):
                w.set_voxel(x, y, z, MAT_STONE)
    return w


PILLARS = [(20, 24, 90), (40, 40, 100), (52, 18, 76), (30, 50, 84)]


def floor_pillars(origin_chunk=(0, 0)):
    """accel.rs:606-666: floor + four 3x3 pillars at a window origin, and the
    fan of clean and grazing rays cast at it.  Returns (world, origin, rays)
    where rays is a list of (eye_world, dir)."""
    w = po.World(*DEFAULT_BRICKS)
    wo = (origin_chunk[0] * 32, 0, origin_chunk[1] * 32)
    for z in range(8, 64):
        for x in range(8, 64):
            for y in range(57, 61):
                apply_edit(w, wo[0] + x, wo[1] + y, wo[2] + z, MAT_STONE, wo)
    for px, pz, top in PILLARS:
        for y in range(61, top):
            for dz in range(3):
                for dx in range(3):
                    apply_edit(w, wo[0] + px + dx, wo[1] + y, wo[2] + pz + dz, MAT_STONE, wo)
    base = np.array(wo, np.float32)
    rays = []
    high_eyes = [(6.0, 96.0, 6.0), (70.0, 110.0, 12.0), (34.0, 130.0, 34.0), (12.0, 74.0, 60.0)]
    for eye in high_eyes:
        eye = np.array(eye, np.float32)
        for gz in range(8):
            for gx in range(8):
                target = np.array([12.0 + gx * 6.0, 62.0, 12.0 + gz * 6.0], np.float32)
                rays.append((eye + base, normalize(target - eye)))
    for px, pz, top in PILLARS:
        eye = np.array([f32(px) - f32(16.0), f32(61 + top) * f32(0.5), f32(pz) + f32(1.5)],
                       np.float32)
        for gy in range(3):
            for gz in range(3):
                target = np.array([f32(px), f32(61.0) + f32(top - 61) * f32(0.25 + gy * 0.25),
                                   f32(pz) + f32(0.5) + f32(gz)], np.float32)
                rays.append((eye + base, normalize(target - eye)))
    return w, wo, rays


def local_safe_inv(x):
    return f32(1e30) if abs(x) < f32(1e-8) else f32(1.0) / f32(x)


def ray_box_entry(o, d, v):
    """accel.rs:581-589: t where o + t*d enters voxel v's unit AABB."""
    inv = np.array([local_safe_inv(d[0]), local_safe_inv(d[1]), local_safe_inv(d[2])], np.float32)
    vmin = np.array(v, np.float32)
    t0 = (vmin - o) * inv
    t1 = (vmin + f32(1.0) - o) * inv
    return max(float(np.minimum(t0, t1).max()), 0.0)


def lattice_touch(p, eps=0.02):
    """accel.rs:597-599: coordinates of p lying on a voxel-lattice plane."""
    return sum(1 for x in p if abs(x - round(float(x))) < eps)


def face_normal(face):
    """record face -> outward normal (voxrt.h face convention)."""
    n = [0, 0, 0]
    if face == 0xFF:
        return tuple(n)
    n[face >> 1] = -1 if (face & 1) else 1
    return tuple(n)


def shadow_scene():
    """accel.rs:837-917: floor with a roof slab at y=80 over [24,44)^2, sun
    normalize(0.16, 0.95, 0.11); floor-cell samples classified decisive."""
    w = flat_floor(8, 8, 56)
    rx0, rx1, rz0, rz1 = 24, 44, 24, 44
    for z in range(rz0, rz1):
        for x in range(rx0, rx1):
            w.set_voxel(x, 80, z, MAT_STONE)
    sun = normalize((0.16, 0.95, 0.11))
    samples = []
    for z in range(10, 62):
        for x in range(10, 62):
            o = np.array([f32(x) + f32(0.5), f32(61.02), f32(z) + f32(0.5)], np.float32)
            s = (80.0 - float(o[1])) / float(sun[1])
            hx = float(o[0]) + float(sun[0]) * s
            hz = float(o[2]) + float(sun[2]) * s
            m = 1.5
            under = rx0 + m < hx < rx1 - m and rz0 + m < hz < rz1 - m
            opn = hx < rx0 - m or hx > rx1 + m or hz < rz0 - m or hz > rz1 + m
            samples.append((o, under, opn))
    return w, sun, samples


def stone_blocks() -> po.World:
    """Solid stone blocks with 16-aligned and unaligned faces (uniform tiles
    and bricks reachable from outside), a glass pane and a water pool."""
    w = po.World(*DEFAULT_BRICKS)
    vx, vy, vz = w.voxels
    blocks = [((64, 32, 64), (192, 96, 192), 4), ((200, 20, 100), (251, 77, 163), 3),
              ((100, 96, 210), (130, 140, 250), 18), ((20, 0, 20), (60, 40, 60), 12)]
    arr = w.a["bricks"]
    for (x0, y0, z0), (x1, y1, z1), m in blocks:
        for x in range(x0, x1):
            for z in range(z0, z1):
                for y in range(y0, y1):
                    b = arr[(x >> 2) + (y >> 2) * 128 + (z >> 2) * 128 * 64]
                    vi = (x & 3) + (z & 3) * 4 + (y & 3) * 16
                    b["occupancy"] |= np.uint64(1 << vi)
                    b["materials"][vi] = m
    w.rebuild()
    return w


def pattern_world(kind, seed=0):
    """Smallest legal window (64x16x64 bricks = 256x64x256 voxels) filled
    with a pattern: 'full' stone, a 3D 'checker' of alternating voxels, or
    'sparse' random voxels (5 %) of every material class."""
    bx, by, bz = 64, 16, 64
    x, y, z = np.meshgrid(np.arange(bx * 4), np.arange(by * 4), np.arange(bz * 4), indexing="ij")
    if kind == "full":
        m = np.full(x.shape, 4, np.uint8)
    elif kind == "checker":
        m = np.where((x + y + z) % 2 == 0, 2, 0).astype(np.uint8)
    else:
        rng = np.random.default_rng(seed)
        classes = np.array([1, 2, 3, 4, 12, 14, 18, 25, 30, 31, 33, 35, 36], np.uint8)
        m = np.where(rng.random(x.shape) < 0.05, rng.choice(classes, x.shape), 0).astype(np.uint8)
    w = po.World(bx, by, bz)
    vi = (x & 3) + (z & 3) * 4 + (y & 3) * 16
    bi = (x >> 2) + (y >> 2) * bx + (z >> 2) * bx * by
    mats = w.a["bricks"]["materials"]
    mats[bi.ravel(), vi.ravel()] = m.ravel()
    occ = (mats != 0).astype(np.uint64) << np.arange(64, dtype=np.uint64)
    w.a["bricks"]["occupancy"] = np.bitwise_or.reduce(occ, axis=1)
    w.rebuild()
    return w


def random_world(rng, bx=64, by=16, bz=64):
    """Boxes and scattered voxels of every material class (water, glass,
    foliage, decoration and leaf fringe included) in a bx*by*bz-brick world."""
    VX, VY, VZ = bx * 4, by * 4, bz * 4
    classes = np.array([1, 2, 3, 4, 5, 8, 12, 14, 18, 25, 30, 31, 33, 34, 35, 36, 37], np.uint8)
    m = np.zeros((VX, VY, VZ), np.uint8)
    for _ in range(int(rng.integers(5, 40))):
        lo = rng.integers([0, 0, 0], [VX, VY, VZ])
        size = rng.integers(1, [64, 24, 64])
        hi = np.minimum(lo + size, [VX, VY, VZ])
        m[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = rng.choice(classes)
    sparse = rng.random(m.shape) < rng.uniform(0.0, 0.03)
    m[sparse] = rng.choice(classes, int(sparse.sum()))
    ow = po.World(bx, by, bz)
    x, y, z = np.meshgrid(np.arange(VX), np.arange(VY), np.arange(VZ), indexing="ij")
    vi = (x & 3) + (z & 3) * 4 + (y & 3) * 16
    bi = (x >> 2) + (y >> 2) * bx + (z >> 2) * bx * by
    mats = ow.a["bricks"]["materials"]
    mats[bi.ravel(), vi.ravel()] = m.ravel()
    occ = (mats != 0).astype(np.uint64) << np.arange(64, dtype=np.uint64)
    ow.a["bricks"]["occupancy"] = np.bitwise_or.reduce(occ, axis=1)
    ow.rebuild()
    return ow
