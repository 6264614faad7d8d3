"""Pin the CPU oracle to the reference's own known-answer tests.

The reference (Rust + WGSL) cannot run here, and it publishes no numeric
golden vectors for ray hits.  Its traversal tests are relational; they are
restated below against the two oracle methods:
  O1 = raycast() restatement (src/raycast.rs),
  O2 = hierarchical trace / trace_any restatement (shaders/raymarch.wgsl).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from scenes import (face_normal, flat_floor, floor_pillars, lattice_touch, normalize,
                    ray_box_entry, shadow_scene)

f32 = np.float32
METHOD = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD


def test_flat_floor_surface_height():
    """accel.rs:529-572: near-vertical rays all hit layer y=60, entering its
    top face y=61."""
    w = flat_floor(16, 16, 48)
    p = po.default_params(METHOD)
    d = normalize((0.03, -1.0, 0.017))
    for gz in range(6):
        for gx in range(6):
            eye = np.array([22.0 + gx * 6.0, 120.0, 22.0 + gz * 6.0], np.float32)
            rec, _ = po.trace_one(w, eye, d, p)
            assert rec["flags"] & 1, "O2 missed the floor"
            assert rec["voxel"][1] == 60
            assert abs(float(eye[1] + rec["t"] * d[1]) - 61.0) < 0.05
            assert face_normal(rec["face"]) == (0, 1, 0)
            hit, vox, nrm, _ = po.raycast(w, eye, d)
            assert hit and vox[1] == 60 and nrm == (0, 1, 0)
            te = ray_box_entry(eye, d, vox)
            assert abs(float(eye[1]) + te * float(d[1]) - 61.0) < 0.05


@pytest.mark.parametrize("origin_chunk", [(0, 0), (3, 5)])
def test_floor_pillars_clean_hits_match_raycast(origin_chunk):
    """accel.rs:606-759: clean (non-grazing) first hits of the hierarchical
    trace equal raycast()'s voxel and normal exactly; the shifted origin
    engages the toroidal storage mapping."""
    w, wo, rays = floor_pillars(origin_chunk)
    p = po.default_params(METHOD)
    clean = floor = pillar = grazing = 0
    for eye, d in rays:
        rec, _ = po.trace_one(w, eye, d, p, ro=wo)
        hit, vox, nrm, _ = po.raycast(w, eye, d, wo)
        o2_hit = bool(rec["flags"] & 1)
        if not o2_hit and not hit:
            continue
        cpu_graze = hit and lattice_touch(eye + f32(ray_box_entry(eye, d, vox)) * d) >= 2
        o2_graze = o2_hit and lattice_touch(eye + rec["t"] * d) >= 2
        if o2_hit and hit and tuple(rec["voxel"]) == vox:
            if cpu_graze:
                grazing += 1
            else:
                clean += 1
                assert face_normal(rec["face"]) == nrm
                if vox[1] - wo[1] <= 60:
                    floor += 1
                else:
                    pillar += 1
            continue
        assert cpu_graze or o2_graze, (eye, d, rec, vox)
        grazing += 1
    total = len(rays)
    assert clean > total / 3
    assert floor > 0 and pillar > 0
    assert grazing < clean


def test_shadow_occlusion_matches_raycast():
    """accel.rs:837-917: any-hit occlusion agrees with raycast().is_some() on
    every decisive sample, and the scene really casts a shadow."""
    w, sun, samples = shadow_scene()
    p = po.default_params(METHOD)
    occ_ok = lit_ok = disagree = 0
    for o, under, opn in samples:
        o2_occ, _ = po.trace_any_one(w, o, sun, p)
        cpu_occ = po.raycast(w, o, sun)[0]
        if o2_occ != cpu_occ:
            if under or opn:
                disagree += 1
            continue
        if under and o2_occ:
            occ_ok += 1
        elif opn and not o2_occ:
            lit_ok += 1
    assert disagree == 0
    assert occ_ok > 20 and lit_ok > 20


def test_empty_world_all_miss():
    """accel.rs:920-942"""
    w = po.World(128, 64, 128)
    p = po.default_params(METHOD)
    d = normalize((0.05, -1.0, 0.03))
    for gz in range(8):
        for gx in range(8):
            eye = np.array([20.0 + gx * 30.0, 200.0, 20.0 + gz * 30.0], np.float32)
            rec, _ = po.trace_one(w, eye, d, p)
            assert not (rec["flags"] & 1) and rec["face"] == 0xFF
            assert not po.trace_any_one(w, eye, d, p)[0]
            assert not po.raycast(w, eye, d)[0]


def test_worldgen_deterministic_and_seed_sensitive():
    """tests/worldgen.rs:19-45 restated for the benchmark generator."""
    from voxelg_b200.configs import CONFIGS
    t = CONFIGS["c1"].terrain
    a = po.World(64, 64, 64)
    b = po.World(64, 64, 64)
    a.generate(t, threads=3)
    b.generate(t, threads=1)
    for k in po.World.NAMES:
        assert np.array_equal(a.a[k].view(np.uint8), b.a[k].view(np.uint8)), k
    import dataclasses
    c = po.World(64, 64, 64)
    c.generate(dataclasses.replace(t, seed=t.seed ^ 0x1234), threads=2)
    assert not np.array_equal(a.a["bricks"].view(np.uint8), c.a["bricks"].view(np.uint8))


def test_incremental_masks_equal_rebuild(c1_oracle_world):
    """refresh_masks_for_brick (voxel.rs:879-914) keeps every mask and LUT equal
    to a from-scratch rebuild, through random edits incl. emptying bricks."""
    src = c1_oracle_world
    w = po.World(*src.dims, arrays={k: v.copy() for k, v in src.a.items()})
    rng = np.random.default_rng(7)
    vx, vy, vz = w.voxels
    for _ in range(4000):
        x, y, z = int(rng.integers(vx)), int(rng.integers(vy)), int(rng.integers(vz))
        m = int(rng.choice([0, 0, 2, 3, 4, 12, 30]))
        w.set_voxel(x, y, z, m)
    # carve a whole region to force tile/chunk/L4 empty transitions
    for x in range(0, 70):
        for z in range(0, 70):
            for y in range(0, 256):
                w.set_voxel(x, y, z, 0)
    r = po.World(*w.dims, arrays={k: v.copy() for k, v in w.a.items()})
    r.rebuild()
    for k in ("tile_mask", "chunk_mask", "l4_mask", "brick_uniform", "tile_uniform"):
        assert np.array_equal(w.a[k], r.a[k]), k


def test_lut_early_out_is_exact():
    """The uniform brick/tile early-out returns the entry voxel of a fully
    solid cell, which the per-voxel descent would return at the same
    iteration: records are identical except the early-out flag bit."""
    import voxelg_b200 as vg
    from scenes import stone_blocks
    w = stone_blocks()
    cam = vg.camera_from_pose((300.0, 150.0, 40.0), -0.6, -0.35, 1.2217305, 160, 90)
    a = po.render_frame(w, cam, po.default_params(po.OR_F_L4))[0]
    b = po.render_frame(w, cam, po.default_params(po.OR_F_L4 | po.OR_F_LUT))[0]
    assert (b["flags"] & 2).any()
    bb = b.copy()
    bb["flags"] &= 1
    assert np.array_equal(a.view(np.uint8), bb.view(np.uint8))


def test_l4_skip_is_exact(c1_oracle_world):
    """The L4 / chunk-in-L4 skips change the iteration count only."""
    import voxelg_b200 as vg
    cam = vg.default_camera((128, 64, 128), 160, 90)
    a = po.render_frame(c1_oracle_world, cam, po.default_params(0))[0]
    b = po.render_frame(c1_oracle_world, cam, po.default_params(po.OR_F_L4))[0]
    for f in ("voxel", "face", "mat", "flags"):
        assert np.array_equal(a[f], b[f]), f
    hit = (a["flags"] & 1) == 1
    assert np.allclose(a["t"][hit], b["t"][hit], rtol=0, atol=1e-3)


def test_terrain_primary_agrees_with_raycast(c1_oracle_world):
    """On the benchmark world, plain hierarchical first hits (no beam, t < 400)
    agree with raycast() on every clean hit (src/accel.rs:588-599 rule)."""
    import voxelg_b200 as vg
    w = c1_oracle_world
    cam = vg.default_camera((128, 64, 128), 96, 54)
    p = po.default_params(po.OR_F_L4)
    rec = po.render_frame(w, cam, p)[0]
    c = po.camera_from(cam)
    clean = graze = 0
    for i in range(len(rec)):
        gx, gy = i % 96, i // 96
        d = np.zeros(3, np.float32)
        u = f32((f32(gx) + f32(0.5)) / f32(96.0))
        v = f32((f32(gy) + f32(0.5)) / f32(54.0))
        dd = (po.C.c_float * 3)()
        po.load().or_ray_dir_uv(po.C.byref(c), float(u), float(v), dd)
        d[:] = list(dd)
        eye = np.array(list(c.origin), np.float32)
        hit, vox, nrm, _ = po.raycast(w, eye, d)
        o2 = bool(rec[i]["flags"] & 1)
        if not hit and not o2:
            continue
        if hit and o2 and tuple(rec[i]["voxel"]) == vox and face_normal(rec[i]["face"]) == nrm:
            clean += 1
            continue
        assert hit and o2
        g1 = lattice_touch(eye + f32(ray_box_entry(eye, d, vox)) * d)
        g2 = lattice_touch(eye + rec[i]["t"] * d)
        assert g1 >= 2 or g2 >= 2, (i, rec[i], vox, nrm)
        graze += 1
    assert clean > 1000 and graze < clean / 20


def test_shadow_rays_need_hits(c1_oracle_world):
    import voxelg_b200 as vg
    cam = vg.default_camera((128, 64, 128), 80, 45)
    rec, sh, _, _, _ = po.render_frame(c1_oracle_world, cam,
                                       po.default_params(po.OR_F_L4 | po.OR_F_SHADOW))
    hit = (rec["flags"] & 1) == 1
    assert np.array_equal(sh["traced"] == 1, hit)
    assert 0 < sh["occluded"][hit].mean() < 1


def test_sincos_series_accuracy():
    import math
    lib = po.load()
    s, c = po.C.c_float(), po.C.c_float()
    for x in np.linspace(0.0, 2.4, 97):
        lib.or_sincos(float(x), po.C.byref(s), po.C.byref(c))
        assert abs(s.value - math.sin(float(f32(x)))) < 4e-7
        assert abs(c.value - math.cos(float(f32(x)))) < 4e-7
