"""GPU parity: every CUDA entry point against the CPU oracle, bit-exact
(hit voxel, face, material, flags, t and step count; integer and float
fields compared as raw bytes), through the C ABI of libvoxrt."""
import math

import numpy as np
import pytest

from oracle import pyoracle as po
from scenes import pattern_world, random_world

pytestmark = pytest.mark.gpu

f32 = np.float32
METHOD = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM


@pytest.fixture(scope="module")
def vg():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200
    return voxelg_b200


@pytest.fixture(scope="module")
def dev_c1(vg):
    cfg = vg.CONFIGS["c1"]
    w = vg.DeviceWorld(*cfg.bricks)
    w.generate(cfg.terrain)
    yield w
    w.close()


def upload_oracle(vg, ow):
    w = vg.DeviceWorld(*ow.dims)
    w.upload(ow.a)
    return w


def assert_same_records(got, want, what=""):
    got = np.ascontiguousarray(got).view(po.RECORD)
    want = np.ascontiguousarray(want).view(po.RECORD)
    assert got.shape == want.shape
    bad = np.flatnonzero((got.view(np.uint8).reshape(-1, 24) !=
                          want.view(np.uint8).reshape(-1, 24)).any(axis=1))
    assert bad.size == 0, f"{what}: {bad.size} records differ, first {bad[:5]}: " \
                          f"got {got[bad[:3]]} want {want[bad[:3]]}"


def frame_pair(vg, dw, ow, cam, flags):
    p = vg.default_params(flags)
    rec, sh = vg.render_primary(dw, cam, p)
    import torch
    torch.cuda.synchronize()
    want = po.render_frame(ow, cam, p)
    return vg.records(rec), (vg.shadows(sh) if sh is not None else None), want


def test_device_worldgen_matches_oracle(vg, dev_c1, c1_oracle_world):
    got = dev_c1.download()
    for k in po.World.NAMES:
        assert np.array_equal(got[k].view(np.uint8), c1_oracle_world.a[k].view(np.uint8)), k


def test_upload_download_roundtrip(vg):
    from scenes import stone_blocks
    ow = stone_blocks()
    w = upload_oracle(vg, ow)
    got = w.download()
    for k in po.World.NAMES:
        assert np.array_equal(got[k].view(np.uint8), ow.a[k].view(np.uint8)), k
    w.close()


@pytest.mark.parametrize("flags", [po.OR_F_L4, 0, METHOD, METHOD | po.OR_F_SHADOW,
                                   po.OR_F_L4 | po.OR_F_LUT | po.OR_F_SHADOW])
def test_c1_frame_bit_exact(vg, dev_c1, c1_oracle_world, flags):
    cfg = vg.CONFIGS["c1"]
    cam = vg.default_camera(dev_c1, cfg.width, cfg.height)
    rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dev_c1, c1_oracle_world, cam, flags)
    assert_same_records(rec, wrec, f"c1 flags={flags}")
    assert (rec["flags"] & 1).mean() > 0.3
    if flags & po.OR_F_SHADOW:
        assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))
        assert sh["traced"].sum() == (rec["flags"] & 1).sum()


@pytest.mark.parametrize("res", [(640, 360), (333, 7), (17, 13)])
def test_refill_schedule_bit_exact(vg, dev_c1, c1_oracle_world, res):
    """The persistent per-lane refill kernel gives the oracle's records."""
    cam = vg.default_camera(dev_c1, *res)
    dev_c1.set_persistent(True)
    try:
        for flags in (po.OR_F_L4, METHOD | po.OR_F_SHADOW, po.OR_F_L4 | po.OR_F_SHADOW):
            rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dev_c1, c1_oracle_world, cam, flags)
            assert_same_records(rec, wrec, f"refill {res} flags={flags}")
            if sh is not None:
                assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))
        # repeated launches: the self-resetting work counters start from zero
        p = vg.default_params()
        a = vg.render_primary(dev_c1, cam, p)
        b = vg.render_primary(dev_c1, cam, p)
        import torch
        torch.cuda.synchronize()
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
        s = vg.render_stats(dev_c1, cam, p)
    finally:
        dev_c1.set_persistent(False)
    assert s == vg.render_stats(dev_c1, cam, p)


def test_frame_stats_match_oracle(vg, dev_c1, c1_oracle_world):
    cfg = vg.CONFIGS["c1"]
    cam = vg.default_camera(dev_c1, 320, 180)
    for flags in (po.OR_F_L4, METHOD | po.OR_F_SHADOW):
        p = vg.default_params(flags)
        s = vg.render_stats(dev_c1, cam, p)
        st = po.render_frame(c1_oracle_world, cam, p)[4]
        b = s["beam"][0] + s["primary"][0]
        i = s["beam"][1] + s["primary"][1]
        assert (b, i) == (st.bytes, st.iters), flags
        if flags & po.OR_F_BEAM:
            bst = po.beam_pass(c1_oracle_world, cam)[1]
            assert s["beam"] == (bst.bytes, bst.iters)


@pytest.mark.parametrize("res", [(1, 1), (17, 13), (64, 36), (333, 7)])
def test_odd_resolutions_and_jitter(vg, dev_c1, c1_oracle_world, res):
    cam = vg.default_camera(dev_c1, *res)
    cam.jitter_x, cam.jitter_y = 0.37, -0.21
    rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dev_c1, c1_oracle_world, cam,
                                               METHOD | po.OR_F_SHADOW)
    assert_same_records(rec, wrec, f"res {res}")
    assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))


@pytest.mark.parametrize("pose", [
    ((256.0, 300.0, 256.0), 0.0, -1.5, "above the window looking down"),
    ((-40.0, 120.0, -30.0), 0.8, -0.2, "outside the window"),
    ((256.0, 70.0, 256.0), 1.3, 0.1, "inside terrain"),
    ((600.0, 140.0, 100.0), -2.0, -0.3, "outside, facing in"),
])
def test_camera_poses(vg, dev_c1, c1_oracle_world, pose):
    pos, yaw, pitch, _ = pose
    cam = vg.camera_from_pose(pos, yaw, pitch, math.radians(70), 96, 64)
    for flags in (po.OR_F_L4, METHOD | po.OR_F_SHADOW):
        rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dev_c1, c1_oracle_world, cam, flags)
        assert_same_records(rec, wrec, str(pose))


def test_shifted_window_origin(vg):
    """Toroidal storage: a window origin away from 0 folds world voxels into
    slots (raymarch.wgsl:17-23)."""
    from scenes import floor_pillars
    ow, wo, _ = floor_pillars((3, 5))
    dw = upload_oracle(vg, ow)
    cam = vg.camera_from_pose((wo[0] + 6.0, 96.0, wo[2] + 6.0), 0.78, -0.5, math.radians(70),
                              128, 72, world_origin=wo)
    for flags in (po.OR_F_L4, METHOD | po.OR_F_SHADOW):
        rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dw, ow, cam, flags)
        assert_same_records(rec, wrec, "shifted origin")
        assert (rec["flags"] & 1).any()
    dw.close()


def test_non_power_of_two_world(vg):
    """A world 768 voxels wide (192 x 32 x 128 bricks, x not a power of two)
    under a shifted window: the general toroidal fold of the traversal gives
    the oracle's records for frames, batched rays of every kind and the
    queue."""
    import voxelg_b200.queue as q
    bricks = (192, 32, 128)
    t = vg.TerrainParams(seed=0x5EED_0F_0DD, base_height=50.0, amplitude=24.0, water_level=30)
    dw = vg.DeviceWorld(*bricks)
    dw.generate(t)
    ow = po.World(*bricks)
    ow.generate(t)
    got = dw.download()
    for k in po.World.NAMES:
        assert np.array_equal(got[k].view(np.uint8), ow.a[k].view(np.uint8)), k
    for wo in ((0, 0, 0), (-448, 0, 320), (1216, 0, -192)):
        cam = vg.camera_from_pose((wo[0] + 383.5, 100.0, wo[2] + 250.25), 1.3, -0.35,
                                  math.radians(70), 200, 112, world_origin=wo)
        for flags in (po.OR_F_L4, METHOD, METHOD | po.OR_F_BEAM | po.OR_F_SHADOW):
            rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dw, ow, cam, flags)
            assert_same_records(rec, wrec, f"non-pow2 frame {wo} {flags}")
            if sh is not None:
                assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))
            assert (rec["flags"] & 1).any()
        rng = np.random.default_rng(abs(wo[0]) + 7)
        rays = random_rays(rng, 6000, (768, 128, 512))
        rays["org"] += np.array(wo, np.float32)
        p = vg.default_params(METHOD)
        want = po.trace_batch(ow, rays, p, origin=wo)[0]
        assert_same_records(vg.records(vg.trace(dw, rays, p, origin=wo)), want, "non-pow2 rays")
        _, out, _ = q.run(dw, rays, p, origin=wo)
        assert_same_records(vg.records(out), want, "non-pow2 queue")
    dw.close()


def random_rays(rng, n, vox, kinds=(0, 1, 2)):
    rays = np.zeros(n, po.RAY)
    lo = np.array([-40, -20, -40], np.float32)
    hi = np.array(vox, np.float32) + np.array([40, 60, 40], np.float32)
    rays["org"] = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    # a share of axis-aligned and zero-component directions
    m = rng.random(n) < 0.1
    d[m, rng.integers(0, 3, m.sum())] = 0.0
    m2 = rng.random(n) < 0.05
    d[m2] = np.array([0.0, -1.0, 0.0], np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    rays["dir"] = d
    rays["tmax"] = rng.choice(np.array([8.0, 64.0, 256.0, 480.0, 700.0], np.float32), n)
    rays["kind"] = rng.choice(np.array(kinds, np.uint32), n)
    return rays


def test_trace_kinds_bit_exact(vg, dev_c1, c1_oracle_world):
    from scenes import stone_blocks
    rng = np.random.default_rng(3)
    for ow, dw in ((c1_oracle_world, dev_c1), (stone_blocks(), None)):
        dw_ = dw or upload_oracle(vg, ow)
        rays = random_rays(rng, 20000, ow.voxels)
        for flags in (po.OR_F_L4, METHOD):
            p = vg.default_params(flags)
            got = vg.records(vg.trace(dw_, rays, p))
            want = po.trace_batch(ow, rays, p)[0]
            assert_same_records(got, want, f"kinds flags={flags}")
        if dw is None:
            dw_.close()


def test_degenerate_rays_bit_exact(vg, dev_c1, c1_oracle_world):
    """NaN / Inf / zero / denormal / huge origins and directions, Inf, NaN
    and negative tmax, every kind and the shadow spawn bit: the device gives
    the oracle's records (defined conversions: NaN -> 0, saturation, clamp
    to +-2^30) through vx_trace and through the mixed queue."""
    import voxelg_b200.queue as q
    nan, inf = np.float32(np.nan), np.float32(np.inf)
    origins = [(nan, 100, 100), (100, 100, 100), (inf, 100, 100), (-inf, -inf, -inf),
               (1e30, 100, 100), (256, 300, 256), (0.0, 0.0, 0.0), (511.999, 255.999, 511.999)]
    dirs = [(0, -1, 0), (nan, -1, 0), (0, 0, 0), (inf, -inf, 0), (1, 1, 1), (-1, 0, 0),
            (1e-30, -1e-30, 1e-38), (1e-8, -1.0, 0.0)]
    rays = []
    for o in origins:
        for d in dirs:
            for tmax, kind in ((700.0, 0), (inf, 1), (-5.0, 2), (nan, 3), (64.0, 256),
                               (300.0, 257), (300.0, 258)):
                rays.append((o, d, tmax, kind))
    r = np.zeros(len(rays), po.RAY)
    for i, (o, d, tmax, kind) in enumerate(rays):
        r[i]["org"], r[i]["dir"], r[i]["tmax"], r[i]["kind"] = o, d, tmax, kind
    def canon(rec):
        # a NaN hit distance (NaN origins) has no meaningful payload: x86 and
        # the GPU produce different NaN bit patterns, so compare it as "NaN"
        rec = np.ascontiguousarray(rec).view(po.RECORD).copy()
        rec["t"][np.isnan(rec["t"])] = np.float32(np.nan)
        return rec

    p = vg.default_params(METHOD)
    want, wsh = po.trace_batch(c1_oracle_world, r, p, shadows=True)[:2]
    assert np.isnan(want["t"]).sum() > 0
    got = vg.records(vg.trace(dev_c1, r, p))
    assert_same_records(canon(got), canon(po.trace_batch(c1_oracle_world, r, p)[0]),
                        "vx_trace degenerate")
    _, out, sh = q.run(dev_c1, r, p)
    assert_same_records(canon(vg.records(out)), canon(want), "queue degenerate")
    assert np.array_equal(vg.shadows(sh).view(np.uint8), wsh.view(np.uint8))


def test_raycast_matches_o1(vg, dev_c1, c1_oracle_world):
    rng = np.random.default_rng(5)
    n = 20000
    vox = c1_oracle_world.voxels
    cams = rng.uniform([-20, 40, -20], [vox[0] + 20, 200, vox[2] + 20], size=(n, 3)).astype(np.float32)
    dirs = rng.normal(size=(n, 3)).astype(np.float32)
    dirs[::17] = 0.0                      # zero direction -> None
    dirs[1::23] *= np.float32(1e-20)      # denormal-ish length
    got, hit = vg.raycast_batch(dev_c1, cams, dirs)
    want, whit, _ = po.raycast_batch(c1_oracle_world, cams, dirs)
    assert np.array_equal(hit, whit)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
    assert 0.2 < hit.mean() < 0.95
    # the single-call drop-in
    for i in range(0, 60, 3):
        h = vg.raycast(cams[i], dirs[i], dev_c1)
        assert (h is not None) == bool(whit[i])
        if h is not None:
            assert h.voxel == tuple(want[i]["voxel"]) and h.normal == tuple(want[i]["normal"])


def test_raycast_bench_case(vg, dev_c1, c1_oracle_world):
    """benches/trace.rs:24-40: origin (256, 90, 256), dir normalize(sin a,
    -0.5, cos a), a += 0.013."""
    n = 4096
    a = (np.arange(1, n + 1, dtype=np.float32) * np.float32(0.013)).astype(np.float32)
    dirs = np.stack([np.sin(a), np.full(n, -0.5, np.float32), np.cos(a)], 1).astype(np.float32)
    cams = np.tile(np.array([256.0, 90.0, 256.0], np.float32), (n, 1))
    got, hit = vg.raycast_batch(dev_c1, cams, dirs)
    want, whit, _ = po.raycast_batch(c1_oracle_world, cams, dirs)
    assert np.array_equal(hit, whit) and np.array_equal(got.view(np.uint8), want.view(np.uint8))


def test_reference_patterns_on_gpu(vg):
    """accel.rs:529-942 patterns through the GPU entry points."""
    from scenes import (face_normal, flat_floor, floor_pillars, lattice_touch, normalize,
                        ray_box_entry, shadow_scene)
    # flat floor
    ow = flat_floor(16, 16, 48)
    dw = upload_oracle(vg, ow)
    d = normalize((0.03, -1.0, 0.017))
    rays = np.zeros(36, po.RAY)
    for i in range(36):
        rays[i]["org"] = (22.0 + (i % 6) * 6.0, 120.0, 22.0 + (i // 6) * 6.0)
        rays[i]["dir"] = d
        rays[i]["tmax"] = 700.0
    rec = vg.records(vg.trace(dw, rays, vg.default_params(METHOD)))
    assert (rec["voxel"][:, 1] == 60).all() and (rec["flags"] & 1).all()
    hy = rays["org"][:, 1] + rec["t"] * d[1]
    assert np.abs(hy - 61.0).max() < 0.05
    dw.close()
    # floor + pillars, shifted origin: GPU trace vs GPU raycast on clean hits
    ow, wo, fan = floor_pillars((3, 5))
    dw = upload_oracle(vg, ow)
    rays = np.zeros(len(fan), po.RAY)
    for i, (e, dd) in enumerate(fan):
        rays[i]["org"], rays[i]["dir"], rays[i]["tmax"] = e, dd, 700.0
    rec = vg.records(vg.trace(dw, rays, vg.default_params(METHOD), origin=wo))
    picks, hits = vg.raycast_batch(dw, rays["org"], rays["dir"], origin=wo)
    clean = 0
    for i, (e, dd) in enumerate(fan):
        if hits[i] and (rec[i]["flags"] & 1) and tuple(rec[i]["voxel"]) == tuple(picks[i]["voxel"]):
            if lattice_touch(e + f32(ray_box_entry(e, dd, picks[i]["voxel"])) * dd) < 2:
                clean += 1
                assert face_normal(rec[i]["face"]) == tuple(picks[i]["normal"])
    assert clean > len(fan) / 3
    dw.close()
    # shadow occlusion
    ow, sun, samples = shadow_scene()
    dw = upload_oracle(vg, ow)
    rays = np.zeros(len(samples), po.RAY)
    rays["org"] = np.array([s[0] for s in samples])
    rays["dir"] = sun
    rays["tmax"] = 480.0
    rays["kind"] = 1
    occ = vg.records(vg.trace(dw, rays, vg.default_params(METHOD)))["flags"] & 1
    _, cpu = vg.raycast_batch(dw, rays["org"], np.tile(sun, (len(samples), 1)))
    dec = np.array([u or o for _, u, o in samples])
    assert np.array_equal(occ[dec] == 1, cpu[dec] == 1)
    under = np.array([u for _, u, _ in samples])
    assert occ[under].sum() > 20 and (occ[~under & dec] == 0).sum() > 20
    dw.close()
    # empty world
    dw = vg.DeviceWorld(128, 64, 128)
    cam = vg.camera_from_pose((256.0, 200.0, 256.0), 0.0, -0.7, 1.2, 64, 64)
    rec, sh = vg.render_primary(dw, cam, vg.default_params())
    r = vg.records(rec)
    assert not (r["flags"] & 1).any() and (r["face"] == 0xFF).all()
    dw.close()


def test_apply_dirty_matches_oracle(vg, c1_oracle_world):
    """Incremental device update from dirty bricks (renderer.rs:1345-1394)
    leaves the same pyramid as the host's set_voxel maintenance, and frames
    traced after it match the oracle."""
    src = c1_oracle_world
    hw = vg.HostWorld(*src.dims)
    for k in po.World.NAMES:
        hw.arrays[k][...] = src.a[k].view(hw.arrays[k].dtype)
    hw.rebuild()
    dw = vg.DeviceWorld(*src.dims)
    dw.sync(hw)                 # all-dirty: full upload
    assert hw.dirty_count() == 0
    ow = po.World(*src.dims, arrays={k: v.copy() for k, v in src.a.items()})
    rng = np.random.default_rng(9)
    vx, vy, vz = ow.voxels
    cam = vg.default_camera(dw, 160, 90)
    for rnd in range(3):
        for _ in range(5000):
            x, y, z = int(rng.integers(vx)), int(rng.integers(vy)), int(rng.integers(vz))
            m = int(rng.choice([0, 0, 2, 4, 12]))
            hw.set_voxel(x, y, z, m)
            ow.set_voxel(x, y, z, m)
        # empty a column stack so tiles, chunks and an L4 bit flip
        for x in range(rnd * 64, rnd * 64 + 64):
            for z in range(0, 64):
                for y in range(0, 256, 1):
                    hw.set_voxel(x, y, z, 0)
                    ow.set_voxel(x, y, z, 0)
        assert hw.dirty_count() > 0
        dw.sync(hw)
        got = dw.download()
        for k in po.World.NAMES:
            assert np.array_equal(got[k].view(np.uint8), ow.a[k].view(np.uint8)), (rnd, k)
        rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dw, ow, cam, METHOD | po.OR_F_SHADOW)
        assert_same_records(rec, wrec, f"after edits round {rnd}")
    dw.close()
    hw.close()


def test_apply_dirty_duplicates_last_wins(vg):
    dw = vg.DeviceWorld(64, 16, 64)
    idx = np.array([5, 9, 5], np.uint32)
    b = np.zeros(3, po.BRICK)
    b[0]["occupancy"] = 1
    b[0]["materials"][0] = 4
    b[1]["occupancy"] = np.uint64(0xFFFFFFFFFFFFFFFF)
    b[1]["materials"][:] = 3
    b[2]["occupancy"] = 2
    b[2]["materials"][1] = 2
    dw.apply_dirty(idx, b)
    got = dw.download()
    assert got["bricks"][5]["occupancy"] == 2 and got["bricks"][5]["materials"][1] == 2
    assert got["brick_uniform"][9] == 3 and got["brick_uniform"][5] == 0
    assert got["tile_mask"][1] != 0 and got["tile_mask"][2] != 0
    assert got["chunk_mask"][0] != 0 and got["l4_mask"][0] != 0
    dw.close()


def test_apply_dirty_on_a_stream_is_ordered(vg):
    """vx_world_apply_dirty on a caller's stream returns at once: three
    updates in a row (duplicates within and across them, staging buffers
    reused) on a torch stream, then a frame on that stream and a download on
    the world's own stream, equal the oracle's world after the same updates
    applied in order (last entry wins)."""
    import torch
    rng = np.random.default_rng(77)
    ow = po.World(64, 16, 64)
    dw = vg.DeviceWorld(64, 16, 64)
    dw.upload(ow.a)
    stream = torch.cuda.Stream()
    nb = 64 * 16 * 64
    for r in range(3):
        n = 4000
        idx = rng.integers(0, nb // 4, n).astype(np.uint32)  # many repeats
        b = np.zeros(n, po.BRICK)
        occ = rng.integers(0, 2 ** 63, n, dtype=np.uint64) & rng.integers(0, 2 ** 63, n,
                                                                           dtype=np.uint64)
        b["occupancy"] = occ
        bits = ((occ[:, None] >> np.arange(64, dtype=np.uint64)) & 1).astype(bool)
        mats = rng.integers(1, 5, (n, 64)).astype(np.uint8)
        b["materials"] = np.where(bits, mats, 0)
        full = rng.random(n) < 0.1
        b["occupancy"][full] = np.uint64(0xFFFFFFFFFFFFFFFF)
        b["materials"][full] = 4
        dw.apply_dirty(idx, b, stream=stream.cuda_stream)
        for i in range(n):  # the oracle: in order, so the last entry wins
            ow.a["bricks"][idx[i]] = b[i]
    ow.rebuild()
    cam = vg.camera_from_pose((128.5, 40.2, 128.5), 0.6, -0.35, 1.2, 160, 90)
    p = vg.default_params()
    with torch.cuda.stream(stream):
        rec = torch.empty(160 * 90 * 24, dtype=torch.uint8, device="cuda")
        sh = torch.empty(160 * 90 * 8, dtype=torch.uint8, device="cuda")
        vg.render_primary(dw, cam, p, rec, sh, stream=stream.cuda_stream)
    stream.synchronize()
    got = dw.download()
    for k in ("tile_mask", "chunk_mask", "l4_mask", "brick_uniform", "tile_uniform"):
        assert np.array_equal(got[k], ow.a[k]), k
    assert np.array_equal(got["bricks"].view(np.uint8), ow.a["bricks"].view(np.uint8))
    want, _, _, _, _ = po.render_frame(ow, cam, p)
    assert np.array_equal(rec.cpu().numpy(), want.view(np.uint8))
    dw.close()


def test_render_host_equals_device(vg, dev_c1):
    cam = vg.default_camera(dev_c1, 320, 180)
    p = vg.default_params()
    rec, sh = vg.render_primary(dev_c1, cam, p)
    hrec, hsh = vg.render_primary_host(dev_c1, cam, p)
    assert np.array_equal(vg.records(rec).view(np.uint8), hrec.view(np.uint8))
    assert np.array_equal(vg.shadows(sh).view(np.uint8), hsh.view(np.uint8))
    # pinned host buffers, twice (the banded copies overwrite every byte)
    import torch
    n = 320 * 180
    rp = torch.full((n * 24,), 0xAB, dtype=torch.uint8).pin_memory()
    sp = torch.full((n * 8,), 0xAB, dtype=torch.uint8).pin_memory()
    for _ in range(2):
        vg.render_primary_host(dev_c1, cam, p, rp.numpy().view(vg._lib.RECORD_DTYPE),
                               sp.numpy().view(vg._lib.SHADOW_DTYPE))
        assert np.array_equal(vg.records(rec).view(np.uint8), rp.numpy())
        assert np.array_equal(vg.shadows(sh).view(np.uint8), sp.numpy())


def test_window_origin_y_rejected(vg, dev_c1):
    """Storage y is world y: a window corner with y != 0 is refused by every
    entry point that takes one, before any kernel runs."""
    cam = vg.camera_from_pose((256.0, 200.0, 256.0), 0.0, -0.3, 1.2, 64, 36,
                              world_origin=(0, 64, 0))
    for call in (lambda: vg.render_primary(dev_c1, cam, vg.default_params()),
                 lambda: vg.render_primary_host(dev_c1, cam, vg.default_params()),
                 lambda: vg.trace(dev_c1, np.zeros(4, po.RAY), vg.default_params(),
                                  origin=(0, 4, 0))):
        with pytest.raises(vg._lib.VxError) as e:
            call()
        assert e.value.code == vg._lib.VX_ERR_INVALID


def test_c2_full_frame_bit_exact(vg):
    """The full benchmark workload: 2048x256x2048 world, 1920x1080 primary
    rays with beam/LUT/LOD, one shadow ray per hit."""
    import torch
    cfg = vg.CONFIGS["c2"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    ow = po.World(*cfg.bricks)
    ow.generate(cfg.terrain)
    got = dw.download()
    for k in po.World.NAMES:
        assert np.array_equal(got[k].view(np.uint8), ow.a[k].view(np.uint8)), k
    del got
    cam = vg.default_camera(dw, cfg.width, cfg.height)
    p = vg.default_params(cfg.flags)
    rec, sh = vg.render_primary(dw, cam, p)
    torch.cuda.synchronize()
    wrec, wsh, _, _, _ = po.render_frame(ow, cam, p)
    assert_same_records(vg.records(rec), wrec, "c2")
    assert np.array_equal(vg.shadows(sh).view(np.uint8), wsh.view(np.uint8))
    r = vg.records(rec)
    assert (r["flags"] & 2).any(), "LOD / uniform early-outs never fired"
    dw.set_persistent(True)
    rec2, sh2 = vg.render_primary(dw, cam, p)
    torch.cuda.synchronize()
    assert torch.equal(rec, rec2) and torch.equal(sh, sh2), "refill schedule differs"
    dw.close()


def test_invalid_calls_fail_loudly(vg, dev_c1):
    from voxelg_b200 import _lib as L
    import ctypes as C
    lib = L.load()
    cam = vg.default_camera(dev_c1, 16, 16)
    cam.res_x = 0.0
    p = vg.default_params()
    rc = lib.vx_render_primary(dev_c1.handle, C.byref(cam), C.byref(p), C.c_void_p(8),
                               C.c_void_p(0), C.c_void_p(0))
    assert rc == L.VX_ERR_INVALID
    idx = np.array([10 ** 9], np.uint32)
    with pytest.raises(L.VxError):
        dev_c1.apply_dirty(idx, np.zeros(1, po.BRICK))


def test_host_frame_pipeline_bit_exact(vg, dev_c1, c1_oracle_world):
    """vx_render_primary_host_async: three frames of different cameras in
    flight into three host buffer pairs (two device buffers alternate), each
    equal to its own oracle frame after vx_render_host_wait."""
    import torch
    cfg = vg.CONFIGS["c1"]
    p = vg.default_params(METHOD | po.OR_F_SHADOW)
    cams = [vg.camera_from_pose((256.0 + 40 * i, 140.0, 256.0 - 30 * i), 0.3 * i, -0.26, 1.22,
                                cfg.width, cfg.height, (0, 0, 0)) for i in range(3)]
    n = cfg.width * cfg.height
    bufs = [(torch.empty(n * 24, dtype=torch.uint8).pin_memory(),
             torch.empty(n * 8, dtype=torch.uint8).pin_memory()) for _ in cams]
    for cam, (r, s) in zip(cams, bufs):
        vg.render_primary_host_async(dev_c1, cam, p, r.numpy().view(po.RECORD),
                                     s.numpy().view(po.SHADOW))
    vg.render_host_wait(dev_c1)
    for cam, (r, s) in zip(cams, bufs):
        wrec, wsh, _, _, _ = po.render_frame(c1_oracle_world, cam, p)
        assert_same_records(r.numpy().view(po.RECORD), wrec, "pipelined host frame")
        assert np.array_equal(s.numpy(), wsh.view(np.uint8))


@pytest.mark.parametrize("kind", ["full", "checker", "sparse"])
def test_pattern_worlds_bit_exact(vg, kind):
    """Extreme worlds: every level uniform (full), the densest voxel-level
    stepping (checker), and every material class scattered (sparse), with
    the camera inside the world; frames under two flag sets and 4k random
    rays of each kind against the oracle."""
    ow = pattern_world(kind)
    dw = upload_oracle(vg, ow)
    for pose in [((128.5, 30.2, 128.5), 0.4, -0.3), ((3.0, 63.0, 250.0), 2.2, -0.9)]:
        cam = vg.camera_from_pose(pose[0], pose[1], pose[2], 1.2, 96, 54)
        for flags in (METHOD | po.OR_F_SHADOW, po.OR_F_L4):
            rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dw, ow, cam, flags)
            assert_same_records(rec, wrec, f"{kind} flags={flags}")
            if sh is not None:
                assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))
    rng = np.random.default_rng(7)
    n = 4000
    rays = np.zeros(n, po.RAY)
    rays["org"] = rng.uniform([-20, -10, -20], [276, 74, 276], (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    rays["dir"] = d
    rays["tmax"] = rng.uniform(1, 400, n).astype(np.float32)
    for kind_id in (0, 1, 2):
        rays["kind"] = kind_id
        p = vg.default_params(METHOD)
        got = vg.records(vg.trace(dw, rays, p))
        want = po.trace_batch(ow, rays, p)[0]
        assert_same_records(got, want, f"{kind} ray kind {kind_id}")
    dw.close()


def test_single_call_pick_matches_o1(vg, dev_c1, c1_oracle_world):
    """The single-ray drop-in (one warp walks one ray 32 voxels at a time):
    3000 calls -- random starts in and around the window (inside terrain,
    in the air, outside), zero, denormal and axis-aligned directions, long
    grazing rays and the criterion picking rays -- each equal to O1."""
    rng = np.random.default_rng(11)
    vox = c1_oracle_world.voxels
    n = 2600
    cams = rng.uniform([-40, -10, -40], [vox[0] + 40, 260, vox[2] + 40], size=(n, 3))
    dirs = rng.normal(size=(n, 3))
    dirs[::13] = 0.0
    dirs[1::29] *= 1e-20
    dirs[2::31] = (1.0, 0.0, 0.0)
    dirs[3::37] = (0.0, -1.0, 0.0)
    dirs[4::41] = (0.0, 0.0, -1.0)
    dirs[5::7, 1] = 1e-3                     # nearly horizontal: long walks
    a = (np.arange(1, 401) * np.float32(0.013)).astype(np.float32)
    bench_dirs = np.stack([np.sin(a), np.full(400, -0.5, np.float32), np.cos(a)], 1)
    cams = np.concatenate([cams, np.tile([256.0, 90.0, 256.0], (400, 1))]).astype(np.float32)
    dirs = np.concatenate([dirs, bench_dirs]).astype(np.float32)
    want, whit, _ = po.raycast_batch(c1_oracle_world, cams, dirs)
    long_walks = 0
    for i in range(len(cams)):
        h = vg.raycast(cams[i], dirs[i], dev_c1)
        assert (h is not None) == bool(whit[i]), i
        if h is not None:
            assert h.voxel == tuple(want[i]["voxel"]) and h.normal == tuple(want[i]["normal"]), i
        if whit[i] and np.abs(np.array(want[i]["voxel"], np.float64) - cams[i]).sum() > 64:
            long_walks += 1
    assert 0.2 < whit.mean() < 0.95 and long_walks > 50


def test_rebuild_in_place_grow_shrink_stream(vg):
    """accel.rs:761-835 (accel_rebuild_in_place_matches_cpu): a 3x3 pillar
    raised on the flat floor through the edit path, removed again, then a
    streamed window origin.  After each in-place update the device arrays
    equal the oracle's, the probe rays' records and picks equal the
    oracle's, and the removed pillar leaves nothing behind."""
    from scenes import MAT_STONE, flat_floor, normalize
    ow = flat_floor(8, 8, 56)
    dw = upload_oracle(vg, ow)
    p = vg.default_params(METHOD)

    def probe(world, eyes, d, wo=(0, 0, 0)):
        rays = np.zeros(len(eyes), po.RAY)
        rays["org"] = np.asarray(eyes, np.float32) + np.asarray(wo, np.float32)
        rays["dir"] = d
        rays["tmax"] = 700.0
        got = vg.records(vg.trace(dw, rays, p, origin=wo))
        assert_same_records(got, po.trace_batch(world, rays, p, origin=wo)[0])
        dirs = np.tile(np.asarray(d, np.float32), (len(eyes), 1))
        picks, hits = vg.raycast_batch(dw, rays["org"], dirs, origin=wo)
        wpicks, whits, _ = po.raycast_batch(world, rays["org"], dirs, origin=wo)
        assert np.array_equal(hits, whits)
        assert np.array_equal(picks.view(np.uint8), wpicks.view(np.uint8))
        return got, picks, hits

    def world_equal(world):
        got = dw.download()
        for k in po.World.NAMES:
            assert np.array_equal(got[k].view(np.uint8), world.a[k].view(np.uint8)), k

    pillar = [(30 + dx, y, 30 + dz) for y in range(61, 75) for dz in range(3) for dx in range(3)]
    eyes = [(20.0, 70.0, 31.5), (20.0, 62.5, 30.2), (20.0, 74.9, 32.9), (20.0, 75.1, 31.0)]
    # grow in place
    for x, y, z in pillar:
        dw.apply_edit(x, y, z, MAT_STONE)
        ow.set_voxel(x, y, z, MAT_STONE)
    world_equal(ow)
    rec, picks, hits = probe(ow, eyes, (1.0, 0.0, 0.0))
    assert hits[:3].all() and not hits[3]
    assert tuple(picks[0]["voxel"]) == (30, 70, 31) and tuple(picks[0]["normal"]) == (-1, 0, 0)
    assert (rec["flags"][:3] & 1).all()
    # shrink in place: the same rays sail over the floor and miss
    for x, y, z in pillar:
        dw.apply_edit(x, y, z, 0)
        ow.set_voxel(x, y, z, 0)
    world_equal(ow)
    rec, picks, hits = probe(ow, eyes, (1.0, 0.0, 0.0))
    assert not hits.any() and not (rec["flags"] & 1).any()
    # streamed: a generated window shifted by (2, 3) chunks
    dw.clear_edits()
    seed = 0xC0FFEE_F00D_BEEF
    dw.fill_window(seed, 0, 0)
    dw.shift_origin(2, 3)
    sw = po.World(*ow.dims)
    po.fill_window(sw, seed, 2, 3)
    world_equal(sw)
    wo = (64, 0, 96)
    rng = np.random.default_rng(3)
    eyes = np.concatenate([[(40.0, 140.0, 40.0)],
                           rng.uniform([8, 100, 8], [500, 200, 500], (63, 3))]).astype(np.float32)
    rec, picks, hits = probe(sw, eyes, normalize((0.001, -1.0, 0.001)), wo)
    assert hits.mean() > 0.9
    cam = vg.camera_from_pose((200.0 + wo[0], 150.0, 300.0 + wo[2]), 0.7, -0.5, 1.2, 96, 54,
                              world_origin=wo)
    got = vg.render_primary(dw, cam, p)[0]
    assert_same_records(vg.records(got), po.render_frame(sw, cam, p)[0], "streamed")
    dw.close()


def test_empty_and_single_item_batches(vg, dev_c1, c1_oracle_world):
    """Zero and one item through every batched entry point, and the smallest
    frames: nothing is launched for an empty batch, a single item equals the
    oracle, 1x1 and 1x2 frames trace like any pixel."""
    import torch
    from voxelg_b200 import queue as q
    ow = c1_oracle_world
    p = vg.default_params(METHOD)
    one = np.zeros(1, po.RAY)
    one["org"] = (100.5, 150.25, 300.75)
    one["dir"] = (0.3, -0.8, 0.52)
    one["dir"] /= np.float32(math.sqrt(float((one["dir"][0] ** 2).sum())))
    one["tmax"] = 700.0
    for kind in (0, 1, 2):
        one["kind"] = kind
        assert len(vg.records(vg.trace(dev_c1, np.zeros(0, po.RAY), p))) == 0
        assert_same_records(vg.records(vg.trace(dev_c1, one, p)), po.trace_batch(ow, one, p)[0],
                            f"one ray kind {kind}")
    picks, hits = vg.raycast_batch(dev_c1, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32))
    assert len(picks) == 0 and len(hits) == 0
    picks, hits = vg.raycast_batch(dev_c1, one["org"], one["dir"])
    wp, wh, _ = po.raycast_batch(ow, one["org"], one["dir"])
    assert np.array_equal(hits, wh) and np.array_equal(picks.view(np.uint8), wp.view(np.uint8))
    p_sh = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_SHADOW)
    one["kind"] = 0
    for rays in (np.zeros(0, po.RAY), one):
        for so in (0, 1):
            t = q.default_tuning()
            t.sort = so
            _, out, sh = q.run(dev_c1, rays, p_sh, tuning=t)
            torch.cuda.synchronize()
            want, wsh, _, _ = po.trace_batch(ow, rays, p_sh, shadows=True)
            assert np.array_equal(out.cpu().numpy(), want.view(np.uint8)), (len(rays), so)
            assert np.array_equal(sh.cpu().numpy(), wsh.view(np.uint8)), (len(rays), so)
    dev_c1.apply_dirty(np.zeros(0, np.uint32), np.zeros(0, po.BRICK))
    for w, h in ((1, 1), (1, 2), (2, 1), (9, 7)):
        cam = vg.camera_from_pose((256.0, 140.0, 256.0), 0.4, -0.3, 1.2, w, h)
        rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dev_c1, ow, cam, METHOD | po.OR_F_SHADOW)
        assert_same_records(rec, wrec, f"{w}x{h} frame")
        assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))


@pytest.mark.parametrize("seed", range(12))
def test_random_worlds_bit_exact(vg, seed):
    """Seeded random worlds (boxes and scattered voxels of every material
    class, water, glass, foliage, decoration and leaf fringe included), a
    random window origin, flag set and camera: the frame, rays of the three
    kinds (degenerate ones among them) and picks equal the oracle's."""
    rng = np.random.default_rng(1000 + seed)
    ow = random_world(rng)
    VX, VY, VZ = ow.voxels
    dw = upload_oracle(vg, ow)
    wo = (int(rng.integers(-3, 4)) * 32 + int(rng.integers(0, 32)), 0,
          int(rng.integers(-3, 4)) * 32 + int(rng.integers(0, 32)))
    flags = int(rng.choice([METHOD, METHOD | po.OR_F_SHADOW, po.OR_F_L4 | po.OR_F_LUT,
                            po.OR_F_LOD | po.OR_F_SHADOW, 0]))
    p = vg.default_params(flags)
    pos = (wo[0] + float(rng.uniform(-20, VX + 20)), float(rng.uniform(5, 120)),
           wo[2] + float(rng.uniform(-20, VZ + 20)))
    cam = vg.camera_from_pose(pos, float(rng.uniform(0, 6.28)), float(rng.uniform(-1.2, 0.6)),
                              1.2, 80, 45, world_origin=wo)
    rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dw, ow, cam, flags)
    assert_same_records(rec, wrec, f"seed {seed} frame")
    if sh is not None:
        assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))
    n = 3000
    rays = np.zeros(n, po.RAY)
    rays["org"] = (np.array(wo, np.float64) + rng.uniform([-40, -20, -40], [VX + 40, VY + 60, VZ + 40],
                                                         (n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[::29] = 0.0
    d[1::31, 1] = 0.0
    d[2::37] *= np.float32(1e-9)
    rays["dir"] = d
    rays["tmax"] = rng.uniform(0.5, 900, n).astype(np.float32)
    for kind in (0, 1, 2):
        rays["kind"] = kind
        got = vg.records(vg.trace(dw, rays, p, origin=wo))
        assert_same_records(got, po.trace_batch(ow, rays, p, origin=wo)[0], f"seed {seed} kind {kind}")
    picks, hits = vg.raycast_batch(dw, rays["org"], d, origin=wo)
    wp, wh, _ = po.raycast_batch(ow, rays["org"], d, origin=wo)
    assert np.array_equal(hits, wh) and np.array_equal(picks.view(np.uint8), wp.view(np.uint8))
    # the same rays as one mixed queue: kinds shuffled, some kind-0 rays spawning
    # a shadow ray at their hit, sorted and unsorted
    import torch
    from voxelg_b200 import _lib as L
    from voxelg_b200 import queue as q
    kinds = rng.integers(0, 3, n).astype(np.uint32)
    kinds[(kinds == 0) & (rng.random(n) < 0.5)] |= np.uint32(L.VX_RAY_SPAWN_SHADOW)
    rays["kind"] = kinds
    pq = vg.default_params(flags | po.OR_F_SHADOW)
    want, wsh, _, _ = po.trace_batch(ow, rays, pq, origin=wo, shadows=True)
    for so in (0, 1):
        t = q.default_tuning()
        t.sort = so
        _, out, qsh = q.run(dw, rays, pq, tuning=t, origin=wo)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want.view(np.uint8)), f"seed {seed} queue sort={so}"
        assert np.array_equal(qsh.cpu().numpy(), wsh.view(np.uint8)), f"seed {seed} shadows sort={so}"
    dw.close()


@pytest.mark.parametrize("seed", range(6))
def test_random_worlds_ao_and_learned(vg, seed):
    """On seeded random worlds with a chunk-aligned window: contact AO of the
    frame's hits equals the oracle's, and the learned form's verification
    walk and restart (no network) give the plain frame's records but for
    steps."""
    import torch
    from voxelg_b200 import learned as vl
    rng = np.random.default_rng(5000 + seed)
    ow = random_world(rng)
    VX, VY, VZ = ow.voxels
    dw = upload_oracle(vg, ow)
    wo = (int(rng.integers(-2, 3)) * 64, 0, int(rng.integers(-2, 3)) * 64)
    pos = (wo[0] + float(rng.uniform(0, VX)), float(rng.uniform(20, 120)), wo[2] + float(rng.uniform(0, VZ)))
    cam = vg.camera_from_pose(pos, float(rng.uniform(0, 6.28)), float(rng.uniform(-1.2, 0.3)),
                              1.2, 96, 54, world_origin=wo)
    flags = METHOD | po.OR_F_SHADOW
    rec, sh, (wrec, _, _, _, _) = frame_pair(vg, dw, ow, cam, flags)
    assert_same_records(rec, wrec, f"seed {seed} frame")
    p = vg.default_params(flags)
    rt, _ = vg.render_primary(dw, cam, p)
    ao = vg.render_ao(dw, cam, rt).cpu().numpy()
    assert np.array_equal(ao.view(np.uint32), po.render_ao(ow, cam, wrec).view(np.uint32))
    for fl in (po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD, 0):
        pl = vg.default_params(fl)
        plain, _ = vg.render_primary(dw, cam, pl)
        out = torch.empty_like(plain)
        st = vl.render_learned(dw, None, cam, pl, out)
        a, b = vg.records(plain).copy(), vg.records(out).copy()
        a["steps"] = 0
        b["steps"] = 0
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (seed, fl)
        assert st.rays == 96 * 54
    dw.close()


@pytest.mark.parametrize("seed", range(4))
def test_random_worlds_edits_keep_the_walk_exact(vg, seed):
    """Rounds of edits on seeded random worlds: random voxels through
    vx_world_apply_edit, then a slab of whole bricks emptied through
    vx_world_apply_dirty so that tile, chunk and L4 bits flip.  After every
    round the device arrays equal the oracle's after the same changes, and so
    does a frame (the per-tile skip words follow the masks)."""
    rng = np.random.default_rng(9000 + seed)
    ow = random_world(rng)
    VX, VY, VZ = ow.voxels
    bx, by, bz = ow.dims
    dw = upload_oracle(vg, ow)
    classes = np.array([0, 0, 0, 2, 4, 12, 14, 18, 33, 35], np.uint8)
    cam = vg.camera_from_pose((VX / 2 + 0.3, 90.0, VZ / 2 + 0.7), float(rng.uniform(0, 6.28)),
                              -0.5, 1.2, 96, 54)
    for rnd in range(4):
        for _ in range(300):
            x, y, z = int(rng.integers(VX)), int(rng.integers(VY)), int(rng.integers(VZ))
            m = int(rng.choice(classes))
            dw.apply_edit(x, y, z, m)
            ow.set_voxel(x, y, z, m)
        # a slab of empty bricks, 16 bricks (one chunk) wide in x and z, all heights
        b0x, b0z = int(rng.integers(0, bx - 16)), int(rng.integers(0, bz - 16))
        gx, gy, gz = np.meshgrid(np.arange(b0x, b0x + 16), np.arange(by), np.arange(b0z, b0z + 16),
                                 indexing="ij")
        idx = (gx + gy * bx + gz * bx * by).astype(np.uint32).ravel()
        dw.apply_dirty(idx, np.zeros(len(idx), po.BRICK))
        ow.a["bricks"][idx] = np.zeros(len(idx), po.BRICK)
        ow.rebuild()
        got = dw.download()
        for k in po.World.NAMES:
            assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8),
                                  np.ascontiguousarray(ow.a[k]).view(np.uint8)), (seed, rnd, k)
        rec, sh, (wrec, wsh, _, _, _) = frame_pair(vg, dw, ow, cam, METHOD | po.OR_F_SHADOW)
        assert_same_records(rec, wrec, f"seed {seed} round {rnd}")
        assert np.array_equal(sh.view(np.uint8), wsh.view(np.uint8))
    dw.close()
