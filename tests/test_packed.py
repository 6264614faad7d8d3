"""Packed host frames: VxPackedRecord (16 bytes per pixel) and
vx_unpack_records.

The packed form carries a pixel's VxHitRecord and VxShadowRecord without
loss: the hit voxel as an index relative to the window corner, face /
material / flags and the two shadow bits, t, and the primary and shadow step
counts in 16 bits each.  Unpacking must give back, byte for byte, the records
vx_render_primary_host writes (the record contract of Hit,
shaders/raymarch.wgsl:378-389, with this library's step and shadow fields).
"""
import ctypes as C
import math

import numpy as np
import pytest

from voxelg_b200 import _lib as L


def pack_np(rec, sh, origin, window):
    """The packed layout, restated with numpy (the checker of both ends)."""
    rec = np.ascontiguousarray(rec).view(L.RECORD_DTYPE)
    out = np.zeros(len(rec), L.PACKED_DTYPE)
    hit = (rec["flags"] & 1) != 0
    rel = rec["voxel"].astype(np.int64) - np.asarray(origin, np.int64)
    idx = rel[:, 0] + window[0] * (rel[:, 1] + window[1] * rel[:, 2])
    out["voxel"] = np.where(hit, idx, 0).astype(np.uint32)
    out["face"], out["mat"], out["flags"], out["t"] = rec["face"], rec["mat"], rec["flags"], rec["t"]
    steps = rec["steps"].astype(np.uint32)
    if sh is not None:
        sh = np.ascontiguousarray(sh).view(L.SHADOW_DTYPE)
        out["shadow"] = sh["occluded"] | (sh["traced"] << 1)
        steps = steps | (sh["steps"].astype(np.uint32) << 16)
    out["steps"] = steps
    return out


def _random_records(rng, n, origin, window):
    rec = np.zeros(n, L.RECORD_DTYPE)
    sh = np.zeros(n, L.SHADOW_DTYPE)
    hit = rng.random(n) < 0.7
    rel = np.stack([rng.integers(0, window[k], n) for k in range(3)], axis=1)
    rec["voxel"] = np.where(hit[:, None], rel + np.asarray(origin), 0)
    rec["face"] = np.where(hit, rng.integers(0, 6, n), 255)
    rec["mat"] = np.where(hit, rng.integers(1, 40, n), 0)
    rec["flags"] = np.where(hit, 1 | (rng.integers(0, 2, n) << 1), 0)
    rec["t"] = np.where(hit, rng.random(n).astype(np.float32) * 700, 0)
    rec["steps"] = rng.integers(0, 65536, n)
    traced = hit & (rng.random(n) < 0.8)
    sh["traced"] = traced
    sh["occluded"] = traced & (rng.random(n) < 0.5)
    sh["steps"] = np.where(traced, rng.integers(0, 65536, n), 0)
    return rec, sh


@pytest.mark.parametrize("origin,window", [((0, 0, 0), (512, 256, 512)),
                                           ((-1237, 0, 98304), (2048, 256, 2048)),
                                           ((5, 0, -7), (4096, 256, 4096))])
def test_unpack_inverts_the_packed_layout(origin, window):
    """Host side, no GPU: packing with numpy and vx_unpack_records round-trip
    random records, including the largest window the index allows."""
    rng = np.random.default_rng(sum(window) + origin[0])
    rec, sh = _random_records(rng, 20000, origin, window)
    packed = pack_np(rec, sh, origin, window)
    import voxelg_b200 as vg
    r2, s2 = vg.unpack_records(packed, origin, window)
    assert r2.tobytes() == rec.tobytes()
    assert s2.tobytes() == sh.tobytes()


def test_unpack_arguments():
    lib = L.load()
    wv = (C.c_uint32 * 3)(512, 256, 512)
    assert lib.vx_unpack_records(None, 4, L.i3((0, 0, 0)), wv, None, None) == L.VX_ERR_INVALID
    zero = (C.c_uint32 * 3)(0, 256, 512)
    buf = np.zeros(1, L.PACKED_DTYPE)
    assert lib.vx_unpack_records(C.c_void_p(L.ptr(buf)), 1, L.i3((0, 0, 0)), zero, None,
                                 None) == L.VX_ERR_INVALID
    # only the outputs asked for are written; n = 0 is a no-op
    assert lib.vx_unpack_records(None, 0, L.i3((0, 0, 0)), wv, None, None) == 0


@pytest.fixture(scope="module")
def worlds():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    out = {}
    for name in ("c1", "c2"):
        cfg = vg.CONFIGS[name]
        dw = vg.DeviceWorld(*cfg.bricks)
        dw.generate(cfg.terrain)
        out[name] = (dw, cfg)
    yield out
    for dw, _ in out.values():
        dw.close()


def _full_and_packed(vg, dw, cam, p, asynchronous):
    n = int(cam.res_x) * int(cam.res_y)
    rec = np.empty(n, L.RECORD_DTYPE)
    sh = np.empty(n, L.SHADOW_DTYPE)
    vg.render_primary_host(dw, cam, p, rec, sh)
    if asynchronous:
        packed = np.empty(n, L.PACKED_DTYPE)
        vg.render_primary_host_packed_async(dw, cam, p, packed)
        vg.render_host_wait(dw)
    else:
        packed = vg.render_primary_host_packed(dw, cam, p)
    return rec, sh, packed


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1", "c2"])
@pytest.mark.parametrize("asynchronous", [False, True], ids=["sync", "async"])
def test_packed_frame_unpacks_to_the_full_records(worlds, name, asynchronous):
    import voxelg_b200 as vg
    dw, cfg = worlds[name]
    window = tuple(4 * b for b in cfg.bricks)
    for flags, pose in ((cfg.flags, None), (1 | 2 | 4, None),
                        (cfg.flags, ((window[0] * 0.3, 170.0, window[2] * 0.7), 2.4, -0.35))):
        if pose is None:
            cam = vg.default_camera(dw, cfg.width, cfg.height)
        else:
            cam = vg.camera_from_pose(pose[0], pose[1], pose[2], math.radians(70), cfg.width,
                                      cfg.height)
        p = vg.default_params(flags)
        rec, sh, packed = _full_and_packed(vg, dw, cam, p, asynchronous)
        assert packed.nbytes * 2 == rec.nbytes + sh.nbytes
        assert np.array_equal(packed, pack_np(rec, sh, tuple(cam.world_origin), window))
        r2, s2 = vg.unpack_records(packed, tuple(cam.world_origin), window)
        assert r2.tobytes() == rec.tobytes(), (name, flags)
        if flags & L.VX_F_SHADOW:
            assert s2.tobytes() == sh.tobytes(), (name, flags)
        else:
            assert not s2.view(np.uint8).any()
        assert (rec["flags"] & 1).any()


@pytest.mark.gpu
def test_packed_frame_with_a_shifted_window():
    """A window whose corner is at negative x and large z (golden world
    uniform_shifted): voxel indices are relative to that corner, in the
    packed and the compact form."""
    import voxelg_b200 as vg
    from test_golden import GOLDEN, WORLDS, camera_of, params_of, world_arrays
    fr = next(f for f in GOLDEN["frames"] if f["world"] == "uniform_shifted")
    w = WORLDS["uniform_shifted"]
    dw = vg.DeviceWorld(*w["bricks"])
    try:
        dw.upload(world_arrays(w))
        cam = camera_of(fr["camera"], True)
        p = params_of(fr["params"], True)
        p.flags |= L.VX_F_SHADOW
        window = tuple(4 * b for b in w["bricks"])
        for asynchronous in (False, True):
            rec, sh, packed = _full_and_packed(vg, dw, cam, p, asynchronous)
            r2, s2 = vg.unpack_records(packed, w["origin"], window)
            assert r2.tobytes() == rec.tobytes()
            assert s2.tobytes() == sh.tobytes()
            assert (rec["voxel"][:, 0][(rec["flags"] & 1) != 0] < 0).any()
            # the compact form of the same frame
            rec, sh, compact = _full_and_compact(vg, dw, cam, p, asynchronous)
            r2, s2 = vg.unpack_compact_records(compact, w["origin"], window)
            assert r2.tobytes() == rec.tobytes()
            assert s2.tobytes() == sh.tobytes()
    finally:
        dw.close()


@pytest.mark.gpu
def test_packed_frame_limits(worlds):
    import voxelg_b200 as vg
    dw, cfg = worlds["c1"]
    cam = vg.default_camera(dw, 64, 36)
    for field in ("max_iters", "any_max_iters"):
        p = vg.default_params(cfg.flags)
        setattr(p, field, 70000)
        with pytest.raises(L.VxError) as e:
            vg.render_primary_host_packed(dw, cam, p)
        assert e.value.code == L.VX_ERR_INVALID
        assert b"65535" in L.load().vx_last_error()
    p = vg.default_params(cfg.flags)
    p.max_iters = 65535
    vg.render_primary_host_packed(dw, cam, p)


# ---------------------------------------------------------------- compact
def compact_np(rec, sh, origin, window):
    """The 12-byte VxCompactRecord layout, restated with numpy."""
    rec = np.ascontiguousarray(rec).view(L.RECORD_DTYPE)
    sh = np.ascontiguousarray(sh).view(L.SHADOW_DTYPE)
    hit = (rec["flags"] & 1) != 0
    rel = rec["voxel"].astype(np.int64) - np.asarray(origin, np.int64)
    idx = np.where(hit, rel[:, 0] + window[0] * (rel[:, 1] + window[1] * rel[:, 2]), 0)
    out = np.zeros(len(rec), L.COMPACT_DTYPE)
    early = (rec["flags"].astype(np.uint32) >> 1) & 1
    tb = rec["t"].view(np.uint32)
    face3 = np.where(hit, rec["face"].astype(np.uint32), 7)
    out["w"][:, 0] = (idx.astype(np.uint32) & 0x3FFFFFFF) | (early << 30) | \
        (sh["occluded"].astype(np.uint32) << 31)
    out["w"][:, 1] = (tb & 0x7FFFFFFF) | (sh["traced"].astype(np.uint32) << 31)
    out["w"][:, 2] = (rec["steps"].astype(np.uint32) & 0x7FF) | \
        ((sh["steps"].astype(np.uint32) & 0x3FF) << 11) | (face3 << 21) | \
        (rec["mat"].astype(np.uint32) << 24)
    return out


@pytest.mark.parametrize("origin,window", [((0, 0, 0), (512, 256, 512)),
                                           ((-1237, 0, 98304), (2048, 256, 2048))])
def test_compact_unpack_inverts_the_layout(origin, window):
    """Host side, no GPU: the numpy compact layout and vx_unpack_compact_records
    round-trip random records within the form's limits (11 / 10-bit steps, a
    2^30-voxel window)."""
    import voxelg_b200 as vg
    rng = np.random.default_rng(7 + window[0])
    rec, sh = _random_records(rng, 40000, origin, window)
    rec["steps"] = rng.integers(0, 2048, len(rec))
    sh["steps"] = np.where(sh["traced"] != 0, rng.integers(0, 1024, len(sh)), 0)
    compact = compact_np(rec, sh, origin, window)
    r2, s2 = vg.unpack_compact_records(compact, origin, window)
    assert r2.tobytes() == rec.tobytes()
    assert s2.tobytes() == sh.tobytes()
    lib = L.load()
    wv = (C.c_uint32 * 3)(*window)
    assert lib.vx_unpack_compact_records(None, 4, L.i3(origin), wv, None, None) == L.VX_ERR_INVALID


def _full_and_compact(vg, dw, cam, p, asynchronous):
    n = int(cam.res_x) * int(cam.res_y)
    rec = np.empty(n, L.RECORD_DTYPE)
    sh = np.empty(n, L.SHADOW_DTYPE)
    vg.render_primary_host(dw, cam, p, rec, sh)
    if asynchronous:
        compact = np.empty(n, L.COMPACT_DTYPE)
        vg.render_primary_host_compact_async(dw, cam, p, compact)
        vg.render_host_wait(dw)
    else:
        compact = vg.render_primary_host_compact(dw, cam, p)
    return rec, sh, compact


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1", "c2"])
@pytest.mark.parametrize("asynchronous", [False, True], ids=["sync", "async"])
def test_compact_frame_unpacks_to_the_full_records(worlds, name, asynchronous):
    """12 bytes per pixel, byte-equal to the full records after unpacking, on
    the c1 and c2 frames (the c2 window holds exactly 2^30 voxels)."""
    import voxelg_b200 as vg
    dw, cfg = worlds[name]
    window = tuple(4 * b for b in cfg.bricks)
    for flags, pose in ((cfg.flags, None), (1 | 2 | 4 | L.VX_F_SHADOW, None),
                        (cfg.flags, ((window[0] * 0.3, 170.0, window[2] * 0.7), 2.4, -0.35))):
        if pose is None:
            cam = vg.default_camera(dw, cfg.width, cfg.height)
        else:
            cam = vg.camera_from_pose(pose[0], pose[1], pose[2], math.radians(70), cfg.width,
                                      cfg.height)
        p = vg.default_params(flags)
        rec, sh, compact = _full_and_compact(vg, dw, cam, p, asynchronous)
        assert compact.nbytes * 8 == (rec.nbytes + sh.nbytes) * 3
        assert np.array_equal(compact, compact_np(rec, sh, tuple(cam.world_origin), window))
        r2, s2 = vg.unpack_compact_records(compact, tuple(cam.world_origin), window)
        assert r2.tobytes() == rec.tobytes(), (name, flags)
        assert s2.tobytes() == sh.tobytes(), (name, flags)
        assert (rec["flags"] & 1).any()


@pytest.mark.gpu
def test_compact_frame_limits(worlds):
    import voxelg_b200 as vg
    dw, cfg = worlds["c1"]
    cam = vg.default_camera(dw, 64, 36)
    for field, bad in (("max_iters", 2048), ("any_max_iters", 1024)):
        p = vg.default_params(cfg.flags)
        setattr(p, field, bad)
        with pytest.raises(L.VxError) as e:
            vg.render_primary_host_compact(dw, cam, p)
        assert e.value.code == L.VX_ERR_INVALID
    p = vg.default_params(cfg.flags)
    p.max_iters, p.any_max_iters = 2047, 1023
    out = vg.render_primary_host_compact(dw, cam, p)
    rec = np.empty(64 * 36, L.RECORD_DTYPE)
    sh = np.empty(64 * 36, L.SHADOW_DTYPE)
    vg.render_primary_host(dw, cam, p, rec, sh)
    r2, s2 = vg.unpack_compact_records(out, tuple(cam.world_origin), tuple(4 * b for b in cfg.bricks))
    assert r2.tobytes() == rec.tobytes() and s2.tobytes() == sh.tobytes()
