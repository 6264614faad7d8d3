"""The benchmark workloads (seeded synthetic worlds and cameras).

c1: 8x4x8 chunks of 64^3 voxels (512x256x512), 640x360 primary rays, the
    plain hierarchical DDA (no beam / LUT / LOD).
c2: 32x4x32 chunks (2048x256x2048), another seed, 1920x1080 primary rays with
    LUTs, beam pre-pass and LOD on, plus one shadow ray per hit toward
    normalize(0.3, 0.8, 0.5) jittered in a 0.5-degree cone.
Both: 5-octave fBm heightfield, wavelength 128, amplitude 48 around y=96,
grass top, 3 dirt, stone, water to y=80, caves where 3D value noise
(wavelength 32) > 0.35.  Camera at the window centre, y=140, pitch -15 deg,
yaw 0, vfov 70 deg.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import _lib as L
from .world import TerrainParams


@dataclass(frozen=True)
class WorldConfig:
    name: str
    bricks: tuple
    terrain: TerrainParams
    width: int
    height: int
    flags: int


CONFIGS = {
    "c1": WorldConfig("c1", (128, 64, 128), TerrainParams(seed=0xC0FFEE_F00D_BEEF), 640, 360,
                      L.VX_F_L4),
    "c2": WorldConfig("c2", (512, 64, 512), TerrainParams(seed=0x0000_0B20_0000_2048), 1920,
                      1080, L.VX_F_METHOD | L.VX_F_SHADOW),
}
