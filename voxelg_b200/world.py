"""Worlds: the device-resident pyramid (VxWorld) and the host mirror of
voxelG's World (VxHostWorld), both owned by libvoxrt.

Host layouts are the reference's (src/voxel.rs:296-343): 72-byte bricks,
u64 masks with child bit x + z*4 + y*16, one-byte uniform LUTs.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass(frozen=True)
class TerrainParams:
    """Seeded synthetic terrain (the benchmark worlds)."""
    seed: int
    base_height: float = 96.0
    amplitude: float = 48.0
    inv_wavelength: float = 1.0 / 128.0
    octaves: int = 5
    water_level: int = 80
    cave_inv_wavelength: float = 1.0 / 32.0
    cave_threshold: float = 0.35
    dirt_depth: int = 3

    def to_c(self) -> L.VxTerrainParams:
        return L.VxTerrainParams(self.seed, self.base_height, self.amplitude,
                                 self.inv_wavelength, self.octaves, self.water_level,
                                 self.cave_inv_wavelength, self.cave_threshold, self.dirt_depth)


def dims_counts(bx: int, by: int, bz: int) -> dict:
    """Array sizes of a world (src/world_dims.rs:12-37)."""
    tx, ty, tz = bx // 4, by // 4, bz // 4
    cx, cy, cz = (tx + 3) // 4, (ty + 3) // 4, (tz + 3) // 4
    lx, ly, lz = (cx + 3) // 4, (cy + 3) // 4, (cz + 3) // 4
    return {"bricks": bx * by * bz, "tiles": tx * ty * tz, "chunks": cx * cy * cz,
            "l4": lx * ly * lz, "voxels": (bx * 4, by * 4, bz * 4)}


def empty_arrays(bx: int, by: int, bz: int) -> dict:
    n = dims_counts(bx, by, bz)
    return {
        "bricks": np.zeros(n["bricks"], L.BRICK_DTYPE),
        "tile_mask": np.zeros(n["tiles"], np.uint64),
        "chunk_mask": np.zeros(n["chunks"], np.uint64),
        "l4_mask": np.zeros(n["l4"], np.uint64),
        "brick_uniform": np.zeros(n["bricks"], np.uint8),
        "tile_uniform": np.zeros(n["tiles"], np.uint8),
    }


ARRAY_NAMES = ("bricks", "tile_mask", "chunk_mask", "l4_mask", "brick_uniform", "tile_uniform")


class DeviceWorld:
    """A world pyramid resident on one GPU (replaces the wgpu buffer set that
    Renderer::upload_world keeps in sync, src/renderer.rs:1248-1394)."""

    def __init__(self, bricks_x: int, bricks_y: int, bricks_z: int, device: int = 0):
        self._lib = L.load()
        self.dims = (bricks_x, bricks_y, bricks_z)
        self.device = device
        h = C.c_void_p()
        L.check(self._lib.vx_world_create(C.byref(L.VxWorldDesc(bricks_x, bricks_y, bricks_z,
                                                                 device)), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self._lib.vx_world_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def voxels(self):
        return (self.dims[0] * 4, self.dims[1] * 4, self.dims[2] * 4)

    def counts(self) -> tuple:
        c = (C.c_uint64 * 4)()
        L.check(self._lib.vx_world_counts(self.handle, c))
        return tuple(int(x) for x in c)

    def set_persistent(self, on: bool):
        """Frame kernels as one persistent wave pulling pixel tiles, or one
        CTA per 16x8 pixels (default); results are identical."""
        t = L.VxTuning()
        L.check(self._lib.vx_world_get_tuning(self.handle, C.byref(t)))
        t.persistent = 1 if on else 0
        L.check(self._lib.vx_world_set_tuning(self.handle, C.byref(t)))

    def upload(self, arrays: dict):
        a = {k: np.ascontiguousarray(arrays[k]) for k in ARRAY_NAMES}
        L.check(self._lib.vx_world_upload(self.handle, *[L.ptr(a[k]) for k in ARRAY_NAMES]))

    def download(self) -> dict:
        out = empty_arrays(*self.dims)
        L.check(self._lib.vx_world_download(self.handle, *[L.ptr(out[k]) for k in ARRAY_NAMES]))
        return out

    def generate(self, terrain: TerrainParams):
        t = terrain.to_c()
        L.check(self._lib.vx_world_generate(self.handle, C.byref(t)))

    def fill_window(self, seed: int, origin_cx: int = 0, origin_cz: int = 0):
        """The reference's chunk generator (gen_slot_bricks) over every
        storage-chunk slot of a window whose lower corner is world chunk
        (origin_cx, 0, origin_cz); origin 0 is fill_demo_terrain."""
        L.check(self._lib.vx_world_fill_window(self.handle, C.c_uint64(seed & (2**64 - 1)),
                                               origin_cx, origin_cz))

    def shift_origin(self, origin_cx: int, origin_cz: int) -> int:
        """Slide the window (shift_origin): regenerates the slots whose
        world chunk changes and returns how many."""
        n = C.c_uint32()
        L.check(self._lib.vx_world_shift_origin(self.handle, origin_cx, origin_cz, C.byref(n)))
        return n.value

    def oob(self, clear: bool = True) -> int:
        """First out-of-range world index the checked library met (array id
        << 56 | index), 0 if none; always 0 in libvoxrt.so."""
        v = C.c_uint64(0)
        L.check(self._lib.vx_world_oob(self.handle, C.byref(v), 1 if clear else 0))
        return int(v.value)

    def apply_edit(self, wx: int, wy: int, wz: int, mat: int):
        """A persistent edit at a world voxel (apply_edit): written now when
        inside the window, and replayed into every chunk generated later."""
        L.check(self._lib.vx_world_apply_edit(self.handle, wx, wy, wz, mat))

    def clear_edits(self):
        L.check(self._lib.vx_world_clear_edits(self.handle))

    def save(self, path):
        """Checkpoint the device world (arrays, edit log, window state) to a
        .vxw file."""
        L.check(self._lib.vx_world_save(self.handle, str(path).encode()))

    def load(self, path):
        """Restore a .vxw checkpoint into this world (same dims)."""
        L.check(self._lib.vx_world_load(self.handle, str(path).encode()))

    def gen_chunks(self, seed: int, chunks):
        """Generate the given world chunks ((x, y, z) rows) into their slots."""
        c = np.ascontiguousarray(np.asarray(chunks, dtype=np.int32).reshape(-1, 3))
        L.check(self._lib.vx_world_gen_chunks(self.handle, C.c_uint64(seed & (2**64 - 1)),
                                              L.ptr(c), len(c)))

    def apply_dirty(self, brick_idx: np.ndarray, bricks: np.ndarray, stream: int = 0):
        idx = np.ascontiguousarray(brick_idx, dtype=np.uint32)
        b = np.ascontiguousarray(bricks).view(L.BRICK_DTYPE)
        assert len(idx) == len(b)
        L.check(self._lib.vx_world_apply_dirty(self.handle, L.ptr(idx), L.ptr(b), len(idx),
                                               C.c_void_p(stream)))

    def sync(self, host: "HostWorld", stream: int = 0):
        L.check(self._lib.vx_world_sync(self.handle, host.handle, C.c_void_p(stream)))


class HostWorld:
    """Host mirror of voxelG's World core (src/voxel.rs World): arrays plus
    set_voxel / apply_edit with incremental mask + uniform maintenance and a
    dirty-brick list."""

    def __init__(self, bricks_x: int, bricks_y: int, bricks_z: int):
        self._lib = L.load()
        self.dims = (bricks_x, bricks_y, bricks_z)
        h = C.c_void_p()
        L.check(self._lib.vx_host_world_create(bricks_x, bricks_y, bricks_z, C.byref(h)))
        self.handle = h
        ptrs = [C.c_void_p() for _ in range(6)]
        L.check(self._lib.vx_host_world_arrays(self.handle, *[C.byref(p) for p in ptrs]))
        n = dims_counts(*self.dims)
        sizes = [n["bricks"] * 72, n["tiles"] * 8, n["chunks"] * 8, n["l4"] * 8, n["bricks"],
                 n["tiles"]]
        dts = [L.BRICK_DTYPE, np.uint64, np.uint64, np.uint64, np.uint8, np.uint8]
        self.arrays = {}
        for name, p, size, dt in zip(ARRAY_NAMES, ptrs, sizes, dts):
            raw = np.ctypeslib.as_array((C.c_uint8 * size).from_address(p.value))
            self.arrays[name] = raw.view(dt)

    def close(self):
        if getattr(self, "handle", None):
            self.arrays = {}
            self._lib.vx_host_world_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_voxel(self, x: int, y: int, z: int, mat: int):
        L.check(self._lib.vx_host_world_set_voxel(self.handle, x, y, z, mat))

    def apply_edit(self, wx: int, wy: int, wz: int, mat: int, origin=(0, 0, 0)):
        L.check(self._lib.vx_host_world_apply_edit(self.handle, wx, wy, wz, mat, L.i3(origin)))

    def rebuild(self):
        L.check(self._lib.vx_host_world_rebuild(self.handle))

    def dirty_count(self) -> int:
        return int(L.check(self._lib.vx_host_world_dirty_count(self.handle)))
