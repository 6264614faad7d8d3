"""The reference's storage-chunk generator gen_slot_bricks
(src/voxel.rs:1322-1500): the oracle restatement pinned by the reference's
own worldgen tests (tests/worldgen.rs:19-45) and by structural facts of the
generator's code, then the device generator byte-equal to the oracle on
whole windows, shifted windows and streamed origins."""
import numpy as np
import pytest

from oracle import pyoracle as po

SEED = 0xC0FFEE_F00D_BEEF   # World::new (voxel.rs:382), benches/trace.rs:12
MAT_WATER, MAT_FRINGE = 12, 33
TREE_MATS = {13, 14, 23, 24, 25, 26, 27, 32, 33}


def _bytes(b):
    return b.view(np.uint8)


def _voxel(bricks, dx, dy, dz):
    b = bricks[(dx // 4) + (dy // 4) * 8 + (dz // 4) * 64]
    return int(b["materials"][(dx & 3) + (dz & 3) * 4 + (dy & 3) * 16])


# ------------------------------------------------ reference tests (tests/worldgen.rs)
def test_worldgen_is_deterministic():
    """tests/worldgen.rs:19-26"""
    a = po.gen_slot_bricks(3, 0, 5, SEED)
    b = po.gen_slot_bricks(3, 0, 5, SEED)
    assert np.array_equal(_bytes(a), _bytes(b))


def test_worldgen_depends_on_seed():
    """tests/worldgen.rs:28-37: the surface chunk cy=2 differs between seeds."""
    a = po.gen_slot_bricks(3, 2, 5, 1)
    b = po.gen_slot_bricks(3, 2, 5, 2)
    assert not np.array_equal(_bytes(a), _bytes(b))


def test_worldgen_depends_on_chunk():
    """tests/worldgen.rs:39-45"""
    a = po.gen_slot_bricks(0, 2, 0, 42)
    b = po.gen_slot_bricks(1, 2, 0, 42)
    assert not np.array_equal(_bytes(a), _bytes(b))


# ------------------------------------------------ structure of the generator's code
@pytest.mark.parametrize("chunk", [(3, 0, 5), (3, 2, 5), (0, 2, 0), (-4, 3, 7), (9, 2, -2)])
def test_occupancy_matches_materials(chunk):
    """Brick::set keeps occupancy bit <=> material != 0 (voxel.rs:315-325)."""
    bricks = po.gen_slot_bricks(*chunk, SEED)
    mats = bricks["materials"]
    bits = ((bricks["occupancy"][:, None] >> np.arange(64, dtype=np.uint64)) & 1).astype(bool)
    assert np.array_equal(bits, mats != 0)


@pytest.mark.parametrize("chunk,seed", [((3, 2, 5), SEED), ((0, 1, 0), 42), ((-6, 2, 4), 7)])
def test_columns_follow_sample_terrain(chunk, seed):
    """Every column up to its height is solid unless a cave is carved, and
    caves are carved only below a water column's seal (cave_seal_y is
    i32::MIN without water, so in_water_seal holds at every y,
    voxel.rs:1356-1368); above the terrain only decoration, water and tree
    materials appear."""
    cx, cy, cz = chunk
    bricks = po.gen_slot_bricks(cx, cy, cz, seed)
    y0 = cy * 32
    for dz in range(0, 32, 3):
        for dx in range(0, 32, 3):
            h, wt = po.sample_terrain(cx * 32 + dx, cz * 32 + dz, seed)
            for dy in range(32):
                y = y0 + dy
                m = _voxel(bricks, dx, dy, dz)
                if y <= h and wt == 0:
                    assert m != 0 and m != MAT_WATER, (dx, y, dz, h)
                elif y > h + 2 and y > wt:
                    assert m == 0 or m in TREE_MATS, (dx, y, dz, m)


def test_water_fills_to_sea_level():
    """Columns below sea level fill h+1..64 with water (voxel.rs:1381-1392)."""
    seen = 0
    for z in range(-600, 600, 37):
        for x in range(-600, 600, 41):
            h, wt = po.sample_terrain(x, z, SEED)
            if wt == 0:
                continue
            assert wt == 64 and h < 64
            cx, cz = x // 32, z // 32
            for cy in {(h + 1) // 32, 64 // 32}:
                b = po.gen_slot_bricks(cx, cy, cz, SEED)
                for y in range(max(h + 1, cy * 32), min(64, cy * 32 + 31) + 1):
                    assert _voxel(b, x - cx * 32, y - cy * 32, z - cz * 32) == MAT_WATER
            seen += 1
            if seen >= 4:
                return
    assert seen > 0, "no water column found in the sampled area"


def test_trees_stand_on_their_column():
    """trees_for_chunk places a tree at h + 1 of its column with the type
    its biome allows (voxel.rs:1560-1589); never more than 12 per chunk."""
    n_total = 0
    for cz in range(-3, 3):
        for cx in range(-3, 3):
            trees = po.trees_for_chunk(cx, cz, SEED)
            assert len(trees) <= 12
            for t in trees:
                x, y, z = (int(v) for v in t["base"])
                assert cx * 32 <= x < cx * 32 + 32 and cz * 32 <= z < cz * 32 + 32
                h, wt = po.sample_terrain(x, z, SEED)
                assert y == h + 1 and wt == 0 and h > 65 and h + 22 < 256
                assert int(t["ttype"]) in (0, 1, 2, 3, 4)
            n_total += len(trees)
    assert n_total > 0


def test_trees_reach_neighbour_chunks():
    """The tree pass paints trees of the eight xz neighbours too
    (voxel.rs:1474-1497): an oak or birch based within 3 voxels of its
    chunk's +x edge puts its top canopy (radius 4 or 3) into the next chunk."""
    for cz in range(-4, 4):
        for cx in range(-4, 4):
            for t in po.trees_for_chunk(cx, cz, SEED):
                x, y, z = (int(v) for v in t["base"])
                ttype, h = int(t["ttype"]), int(t["hash"])
                if ttype not in (0, 1, 3) or x - cx * 32 < 29:
                    continue
                top = y + (8 + h % 5)
                vx, ncx = x + 3, cx + 1
                b = po.gen_slot_bricks(ncx, top // 32, cz, SEED)
                m = _voxel(b, vx - ncx * 32, top % 32, z - cz * 32)
                assert m in TREE_MATS, (x, y, z, m)
                return
    pytest.fail("no oak or birch near a chunk edge in the sampled area")


def test_fill_window_places_chunks_toroidally():
    """fill_demo_terrain / shift_origin (voxel.rs:507-537, :1005-1060): slot
    (sx, sy, sz) of a window at origin (ox, oz) holds world chunk
    (ox + pos_mod(sx - ox, SX), sy, oz + pos_mod(sz - oz, SZ))."""
    bx, by, bz = 16, 16, 16
    w = po.World(bx, by, bz)
    ox, oz = 5, -3
    po.fill_window(w, SEED, ox, oz, threads=4)
    sxn, syn, szn = bx // 8, by // 8, bz // 8
    bricks = w.a["bricks"].reshape(bz, by, bx)
    for sz in range(szn):
        for sy in range(syn):
            for sx in range(sxn):
                wcx = ox + (sx - ox) % sxn
                wcz = oz + (sz - oz) % szn
                want = po.gen_slot_bricks(wcx, sy, wcz, SEED).reshape(8, 8, 8)
                got = bricks[sz * 8:sz * 8 + 8, sy * 8:sy * 8 + 8, sx * 8:sx * 8 + 8]
                assert np.array_equal(_bytes(np.ascontiguousarray(got)), _bytes(want))
    # masks rebuilt from the bricks
    ref = po.World(bx, by, bz, {k: v.copy() for k, v in w.a.items()})
    ref.rebuild()
    for k in po.World.NAMES:
        assert np.array_equal(ref.a[k].view(np.uint8), w.a[k].view(np.uint8)), k


# ------------------------------------------------ device generator
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")


def _oracle_window(dims, seed, ox, oz):
    w = po.World(*dims)
    po.fill_window(w, seed, ox, oz)
    return w


def _assert_world_equal(dev, ref):
    got = dev.download()
    for k in po.World.NAMES:
        a = np.ascontiguousarray(got[k]).view(np.uint8)
        b = ref.a[k].view(np.uint8)
        if not np.array_equal(a, b):
            bad = np.flatnonzero(a != b)
            raise AssertionError(f"{k}: {len(bad)} bytes differ, first at {bad[:8]}")


DEMO = (128, 64, 128)   # WORLD_BRICKS_X/Y/Z, world_dims.rs:12-14


@pytest.mark.gpu
@pytest.mark.parametrize("seed,origin", [(SEED, (0, 0)), (0xABCD_1234_5678_9999, (0, 0)),
                                         (42, (3, -2)), (1, (-7, 11))])
def test_device_window_equals_oracle(seed, origin):
    _gpu()
    import voxelg_b200 as vg
    dw = vg.DeviceWorld(*DEMO)
    dw.fill_window(seed, *origin)
    _assert_world_equal(dw, _oracle_window(DEMO, seed, *origin))
    dw.close()


@pytest.mark.gpu
def test_device_streaming_round_trip():
    """shift_origin regenerates only the slots whose chunk changes, and a
    far shift and back reproduces the window (tests/worldgen.rs:47-81
    without the edit log)."""
    _gpu()
    import voxelg_b200 as vg
    dw = vg.DeviceWorld(*DEMO)
    dw.fill_window(SEED, 0, 0)
    n = dw.shift_origin(1, -1)
    assert n == 16 * 8 + 16 * 8 - 8
    _assert_world_equal(dw, _oracle_window(DEMO, SEED, 1, -1))
    assert dw.shift_origin(1, -1) == 0
    assert dw.shift_origin(16, 16) == 16 * 8 * 16
    assert dw.shift_origin(0, 0) == 16 * 8 * 16
    _assert_world_equal(dw, _oracle_window(DEMO, SEED, 0, 0))
    dw.close()


@pytest.mark.gpu
def test_device_gen_chunks_later_wins():
    _gpu()
    import voxelg_b200 as vg
    dw = vg.DeviceWorld(*DEMO)
    dw.fill_window(SEED, 0, 0)
    # (16, 2, 0) and (0, 2, 0) share slot (0, 2, 0); the later one wins
    dw.gen_chunks(SEED, [(0, 2, 0), (16, 2, 0), (5, 3, 33)])
    got = dw.download()["bricks"].reshape(128, 64, 128)
    for (cx, cy, cz) in [(16, 2, 0), (5, 3, 33)]:
        sx, sz = cx % 16, cz % 16
        want = po.gen_slot_bricks(cx, cy, cz, SEED).reshape(8, 8, 8)
        blk = np.ascontiguousarray(got[sz * 8:sz * 8 + 8, cy * 8:cy * 8 + 8, sx * 8:sx * 8 + 8])
        assert np.array_equal(_bytes(blk), _bytes(want))
    dw.close()


@pytest.mark.gpu
def test_device_gen_rejects_bad_chunks():
    _gpu()
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    dw = vg.DeviceWorld(*DEMO)
    for bad in [(0, 8, 0), (0, -1, 0), (1 << 24, 0, 0)]:
        with pytest.raises(L.VxError) as e:
            dw.gen_chunks(SEED, [bad])
        assert e.value.code == L.VX_ERR_INVALID
    with pytest.raises(L.VxError):
        dw.shift_origin(1, 1)      # no window generated yet
    dw.gen_chunks(SEED, [(0, 2, 0)])
    with pytest.raises(L.VxError):
        dw.shift_origin(1, 1)      # a list of chunks is not a window
    dw.fill_window(SEED, 0, 0)
    assert dw.shift_origin(1, 0) == 8 * 16
    c1 = vg.CONFIGS["c1"]
    dw.generate(c1.terrain)        # replaces the world: the slot table is void
    with pytest.raises(L.VxError):
        dw.shift_origin(2, 0)
    dw.close()


@pytest.mark.gpu
def test_device_full_size_window_sampled():
    """The 2048x256x2048 window (32768 chunks, the bench's size): 256
    random slots byte-equal to the oracle's gen_slot_bricks, and the masks
    consistent with the bricks (every occupied brick's tile bit set)."""
    _gpu()
    import voxelg_b200 as vg
    dims = (512, 64, 512)
    ox, oz = -5, 9
    dw = vg.DeviceWorld(*dims)
    dw.fill_window(SEED, ox, oz)
    got = dw.download()
    bricks = got["bricks"].reshape(dims[2], dims[1], dims[0])
    rng = np.random.default_rng(3)
    for sx, sy, sz in zip(rng.integers(0, 64, 256), rng.integers(0, 8, 256),
                          rng.integers(0, 64, 256)):
        cx, cz = ox + (sx - ox) % 64, oz + (sz - oz) % 64
        blk = np.ascontiguousarray(bricks[sz * 8:sz * 8 + 8, sy * 8:sy * 8 + 8,
                                          sx * 8:sx * 8 + 8]).reshape(-1)
        assert np.array_equal(blk.view(np.uint8), po.gen_slot_bricks(cx, sy, cz, SEED)
                              .view(np.uint8)), (sx, sy, sz)
    occ = (bricks["occupancy"] != 0).reshape(dims[2] // 4, 4, dims[1] // 4, 4, dims[0] // 4, 4)
    tiles = got["tile_mask"].reshape(dims[2] // 4, dims[1] // 4, dims[0] // 4)
    assert np.array_equal(occ.any(axis=(1, 3, 5)), tiles != 0)
    dw.close()


@pytest.mark.gpu
def test_device_far_chunks():
    """Chunks far from the origin (|x|, |z| up to 2^20 chunks, 2^25 voxels,
    where float coordinates lose their low bits) equal the oracle's."""
    _gpu()
    import voxelg_b200 as vg
    dw = vg.DeviceWorld(*DEMO)
    far = [(1 << 20, 2, -(1 << 20) + 3), (-777777, 1, 654321), (123457, 2, -98765)]
    dw.gen_chunks(SEED, far)
    got = dw.download()["bricks"].reshape(128, 64, 128)
    for cx, cy, cz in far:
        sx, sz = cx % 16, cz % 16
        blk = np.ascontiguousarray(got[sz * 8:sz * 8 + 8, cy * 8:cy * 8 + 8,
                                       sx * 8:sx * 8 + 8]).reshape(-1)
        assert np.array_equal(blk.view(np.uint8), po.gen_slot_bricks(cx, cy, cz, SEED)
                              .view(np.uint8)), (cx, cy, cz)
    dw.close()


@pytest.mark.gpu
def test_frame_on_reference_world():
    """Primary and shadow rays over the reference's own demo world
    (fill_demo_terrain at seed 0xC0FFEE_F00D_BEEF): trees, leaf fringe and
    decoration exercise the material rules the synthetic worlds lack."""
    _gpu()
    import torch

    import voxelg_b200 as vg
    dw = vg.DeviceWorld(*DEMO)
    dw.fill_window(SEED, 0, 0)
    ow = _oracle_window(DEMO, SEED, 0, 0)
    cam = vg.default_camera(dw, 640, 360)
    method = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM
    for flags in (method | po.OR_F_SHADOW, po.OR_F_L4):
        p = vg.default_params(flags)
        rec, sh = vg.render_primary(dw, cam, p)
        torch.cuda.synchronize()
        wrec, wsh, _, _, _ = po.render_frame(ow, cam, p)
        got = vg.records(rec)
        assert np.array_equal(got.view(np.uint8), wrec.view(np.uint8)), flags
        if sh is not None:
            assert np.array_equal(vg.shadows(sh).view(np.uint8), wsh.view(np.uint8))
        mats = set(np.unique(got["mat"][(got["flags"] & 1) == 1]).tolist())
        assert mats & {14, 25, 26, 27, 33}, mats   # foliage was hit
    dw.close()


def test_hash_normalisation_without_division():
    """The device noise computes hash2/hash3's (h & 0xFFFFFF) / 16777215.0
    (voxel.rs:1180, :1192) as float(u) * 2^-24 with its bit pattern plus
    one: equal to the IEEE binary32 quotient for every u < 2^24."""
    u = np.arange(1 << 24, dtype=np.uint32)
    q = u.astype(np.float32) / np.float32(16777215.0)
    p = (u.astype(np.float32) * np.float32(2.0 ** -24)).view(np.uint32)
    r = np.where(u != 0, p + np.uint32(1), np.uint32(0)).view(np.float32)
    assert np.array_equal(q.view(np.uint32), r.view(np.uint32))


MAT_GLASS = 18


def _material_at_world(dw, origin_c, wx, wy, wz):
    """World::material_at_world for the device window at chunk origin_c."""
    ox, oz = origin_c[0] * 32, origin_c[1] * 32
    vx, vy, vz = dw.dims[0] * 4, dw.dims[1] * 4, dw.dims[2] * 4
    assert ox <= wx < ox + vx and 0 <= wy < vy and oz <= wz < oz + vz
    x, z = wx % vx, wz % vz
    b = dw.download()["bricks"].reshape(dw.dims[2], dw.dims[1], dw.dims[0])[z // 4, wy // 4, x // 4]
    return int(b["materials"][(x & 3) + (z & 3) * 4 + (wy & 3) * 16])


def _oracle_with_edits(seed, origin_c, edits):
    ow = _oracle_window(DEMO, seed, *origin_c)
    vx, vz = DEMO[0] * 4, DEMO[2] * 4
    for (x, y, z), m in edits.items():
        if origin_c[0] * 32 <= x < origin_c[0] * 32 + vx and \
                origin_c[1] * 32 <= z < origin_c[1] * 32 + vz and 0 <= y < DEMO[1] * 4:
            ow.set_voxel(x % vx, y, z % vz, m)
    return ow


@pytest.mark.gpu
def test_device_edits_survive_streaming_round_trip():
    """tests/worldgen.rs:47-81: edits applied in the window survive a shift of
    the whole window away and back (every slot unloaded and regenerated,
    the edit log replayed), and the world equals the oracle's with the same
    edits set."""
    _gpu()
    import voxelg_b200 as vg
    seed = 0xABCD_1234_5678_9999
    dw = vg.DeviceWorld(*DEMO)
    dw.fill_window(seed, 0, 0)
    edits = {(10, 100, 10): MAT_GLASS, (40, 70, 80): MAT_GLASS, (200, 64, 130): MAT_GLASS}
    for (x, y, z), m in edits.items():
        dw.apply_edit(x, y, z, m)
        assert _material_at_world(dw, (0, 0), x, y, z) == MAT_GLASS
    _assert_world_equal(dw, _oracle_with_edits(seed, (0, 0), edits))
    assert dw.shift_origin(16, 16) == 16 * 8 * 16
    assert dw.shift_origin(0, 0) == 16 * 8 * 16
    for (x, y, z) in edits:
        assert _material_at_world(dw, (0, 0), x, y, z) == MAT_GLASS
    _assert_world_equal(dw, _oracle_with_edits(seed, (0, 0), edits))
    dw.close()


@pytest.mark.gpu
def test_device_edits_replayed_when_streamed_in():
    """An edit recorded outside the window is not written, and appears when
    a shift brings its chunk into the window; a clearing edit (material 0)
    empties a terrain voxel and its masks follow."""
    _gpu()
    import voxelg_b200 as vg
    dw = vg.DeviceWorld(*DEMO)
    dw.fill_window(SEED, 0, 0)
    edits = {(600, 90, 20): MAT_GLASS, (100, 10, 100): 0, (-3, 80, 7): MAT_GLASS}
    for (x, y, z), m in edits.items():
        dw.apply_edit(x, y, z, m)
    assert _material_at_world(dw, (0, 0), 100, 10, 100) == 0
    _assert_world_equal(dw, _oracle_with_edits(SEED, (0, 0), edits))
    dw.shift_origin(4, -1)                  # x in [128, 640), z in [-32, 480)
    assert _material_at_world(dw, (4, -1), 600, 90, 20) == MAT_GLASS
    _assert_world_equal(dw, _oracle_with_edits(SEED, (4, -1), edits))
    dw.clear_edits()
    dw.shift_origin(0, 0)
    dw.shift_origin(4, -1)                  # regenerated without the log
    assert _material_at_world(dw, (4, -1), 600, 90, 20) != MAT_GLASS
    _assert_world_equal(dw, _oracle_window(DEMO, SEED, 4, -1))
    dw.close()


@pytest.mark.gpu
def test_full_size_generated_window_frame_bit_exact():
    """The 2048x256x2048 window generated by the reference's generator
    (32768 chunks): every byte of the world equals the oracle's, and a
    1920x1080 frame with beam/LUT/LOD and shadow rays over it is bit-exact."""
    _gpu()
    import torch

    import voxelg_b200 as vg
    dims = (512, 64, 512)
    dw = vg.DeviceWorld(*dims)
    dw.fill_window(SEED, 0, 0)
    ow = po.World(*dims)
    po.fill_window(ow, SEED, 0, 0)
    _assert_world_equal(dw, ow)
    cam = vg.camera_from_pose((1024.0, 150.0, 1024.0), 0.7, -0.3, 1.22, 1920, 1080)
    flags = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM | po.OR_F_SHADOW
    p = vg.default_params(flags)
    rec, sh = vg.render_primary(dw, cam, p)
    torch.cuda.synchronize()
    wrec, wsh, _, _, _ = po.render_frame(ow, cam, p)
    got = vg.records(rec)
    assert np.array_equal(got.view(np.uint8), wrec.view(np.uint8))
    assert np.array_equal(vg.shadows(sh).view(np.uint8), wsh.view(np.uint8))
    assert (got["flags"] & 1).mean() > 0.3
    dw.close()


@pytest.mark.gpu
def test_world_checkpoint_round_trip(tmp_path):
    """vx_world_save / vx_world_load: a streamed, edited window restored into
    a fresh world equals the original, and both stream on identically (edit
    log and slot table come back too); wrong dims and truncated files are
    rejected."""
    _gpu()
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    a = vg.DeviceWorld(*DEMO)
    a.fill_window(SEED, 2, -1)
    a.apply_edit(100, 90, 40, MAT_GLASS)
    a.apply_edit(700, 95, 60, MAT_GLASS)    # outside the window for now
    path = tmp_path / "w.vxw"
    a.save(path)
    b = vg.DeviceWorld(*DEMO)
    b.load(path)

    def same(x, y):
        gx, gy = x.download(), y.download()
        for k in po.World.NAMES:
            assert np.array_equal(np.ascontiguousarray(gx[k]).view(np.uint8),
                                  np.ascontiguousarray(gy[k]).view(np.uint8)), k
    def same_frame(x, y, wo):
        # the restored world traces like the original (its derived per-tile
        # words included)
        cam = vg.camera_from_pose((wo[0] + 256.0, 150.0, wo[2] + 256.0), 0.5, -0.4, 1.2, 128, 72,
                                  world_origin=wo)
        p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM | po.OR_F_SHADOW)
        rx, sx = vg.render_primary(x, cam, p)
        ry, sy = vg.render_primary(y, cam, p)
        assert np.array_equal(vg.records(rx).view(np.uint8), vg.records(ry).view(np.uint8))
        assert np.array_equal(vg.shadows(sx).view(np.uint8), vg.shadows(sy).view(np.uint8))
        assert (vg.records(rx)["flags"] & 1).mean() > 0.3
    same(a, b)
    same_frame(a, b, (64, 0, -32))
    assert a.shift_origin(8, 0) == b.shift_origin(8, 0) > 0
    same(a, b)
    same_frame(a, b, (256, 0, 0))
    assert _material_at_world(b, (8, 0), 700, 95, 60) == MAT_GLASS
    small = vg.DeviceWorld(64, 64, 64)
    with pytest.raises(L.VxError) as e:
        small.load(path)
    assert e.value.code == L.VX_ERR_INVALID
    cut = tmp_path / "cut.vxw"
    cut.write_bytes(path.read_bytes()[:100000])
    with pytest.raises(L.VxError):
        b.load(cut)
    for w in (a, b, small):
        w.close()


@pytest.mark.gpu
def test_frame_far_from_origin():
    """renderer.rs:7612-7630 (renders_far_from_origin): the window streamed
    100,000 chunks from spawn, 3.2M voxels, where an f32 ulp is 0.25 voxel.
    With the origin rebased, the frame and the picks traced there equal the
    oracle's bit for bit and, like the spawn frame, show terrain and sky."""
    _gpu()
    import voxelg_b200 as vg
    flags = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM | po.OR_F_SHADOW
    p = vg.default_params(flags)
    dw = vg.DeviceWorld(*DEMO)
    fractions = []
    for oc in [(0, 0), (100_000, 100_000), (-100_000, 37)]:
        dw.fill_window(SEED, *oc)
        ow = _oracle_window(DEMO, SEED, *oc)
        wo = (oc[0] * 32, 0, oc[1] * 32)
        cam = vg.camera_from_pose((wo[0] + 256.0, 150.0, wo[2] + 256.0), 0.7, -0.3, 1.2, 320, 180,
                                  world_origin=wo)
        rec, sh = vg.render_primary(dw, cam, p)
        want, wsh, _, _, _ = po.render_frame(ow, cam, p)
        got = vg.records(rec)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), oc
        assert np.array_equal(vg.shadows(sh).view(np.uint8), wsh.view(np.uint8)), oc
        fractions.append(float((got["flags"] & 1).mean()))
        rng = np.random.default_rng(oc[0] & 0xFFFF)
        cams = (np.array(wo, np.float64) + rng.uniform([0, 100, 0], [512, 200, 512], (500, 3)))
        cams = cams.astype(np.float32)
        dirs = rng.normal(size=(500, 3)).astype(np.float32)
        picks, hits = vg.raycast_batch(dw, cams, dirs, origin=wo)
        wpicks, whits, _ = po.raycast_batch(ow, cams, dirs, origin=wo)
        assert np.array_equal(hits, whits) and np.array_equal(picks.view(np.uint8),
                                                              wpicks.view(np.uint8)), oc
    # terrain and sky in every frame, far frames like the spawn frame
    assert all(0.2 < f < 0.95 for f in fractions), fractions
    dw.close()
