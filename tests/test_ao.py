"""Contact AO of primary hits (compute_ao, shaders/raymarch.wgsl:4417-4475):
the oracle on crafted scenes whose values follow from the corner rule, and
the device pass bit-exact against the oracle on frames of the benchmark
worlds."""
import math

import numpy as np
import pytest

from oracle import pyoracle as po
import scenes

METHOD = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD


def _down_camera(x, z, y=70.0, res=96):
    """Camera straight down (pitch -89.9 deg) over (x, z)."""
    return po.camera_from_pose((x, y, z), 0.0, math.radians(-89.9), math.radians(30.0), res, res)


def test_open_floor_is_unoccluded():
    w = scenes.flat_floor(100, 100, 64)
    w.rebuild()
    cam = _down_camera(132.5, 132.5)
    rec = po.render_frame(w, cam, po.default_params(METHOD))[0]
    hit = (rec["flags"] & 1) == 1
    assert hit.all() and (rec["voxel"][:, 1] == 60).all()
    assert (po.render_ao(w, cam, rec) == 1.0).all()


def test_block_beside_a_floor_voxel_follows_the_corner_rule():
    """One stone block at (x0+1, 61, z0) beside the floor: on the top face of
    floor voxel (x0, 60, z0) the two +x corners see one side occluder
    (1 - 0.22), the -x corners none, so AO = 1 - 0.22 * frac(x)."""
    x0, z0 = 130, 130
    w = scenes.flat_floor(100, 100, 64)
    w.set_voxel(x0 + 1, 61, z0, scenes.MAT_STONE)
    w.rebuild()
    cam = _down_camera(x0 + 0.5, z0 + 0.5, res=128)
    rec = po.render_frame(w, cam, po.default_params(METHOD))[0]
    ao = po.render_ao(w, cam, rec)
    on = (rec["voxel"][:, 0] == x0) & (rec["voxel"][:, 1] == 60) & (rec["voxel"][:, 2] == z0)
    assert on.sum() > 20
    W = 128
    idx = np.nonzero(on)[0]
    for i in idx:
        px, py = i % W, i // W
        d = np.zeros(3, np.float32)
        cc = po.camera_from(cam)
        u = (np.float32(px) + np.float32(0.5)) / np.float32(W)
        v = (np.float32(py) + np.float32(0.5)) / np.float32(W)
        po.load().or_ray_dir_uv(po.C.byref(cc), float(u), float(v),
                                d.ctypes.data_as(po.C.POINTER(po.C.c_float)))
        fx = (np.float32(cc.origin[0]) + d[0] * rec["t"][i]) - np.float32(x0)
        want = 1.0 - 0.22 * min(max(float(fx), 0.0), 1.0)
        assert ao[i] == pytest.approx(want, abs=2e-6), (i, ao[i], want)
    # the block's own top face is open on every side: unoccluded
    top = (rec["voxel"][:, 0] == x0 + 1) & (rec["voxel"][:, 1] == 61) & (rec["face"] == 2)
    assert top.any() and (ao[top] == 1.0).all()


def test_skip_rule_beyond_ao_distance():
    """Hits beyond 64 voxels keep AO = 1 (raymarch.wgsl:3862)."""
    x0, z0 = 130, 130
    w = scenes.flat_floor(100, 100, 64)
    for dz in range(-2, 3):
        w.set_voxel(x0 + 1, 61, z0 + dz, scenes.MAT_STONE)
    w.rebuild()
    near = _down_camera(x0 + 0.5, z0 + 0.5, y=120.0)
    far = _down_camera(x0 + 0.5, z0 + 0.5, y=130.0)
    for cam, expect_any_occluded in ((near, True), (far, False)):
        rec = po.render_frame(w, cam, po.default_params(METHOD))[0]
        ao = po.render_ao(w, cam, rec)
        assert ((ao < 1.0).any()) == expect_any_occluded


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def c1(c1_oracle_world):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200 as vg
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    yield vg, dw
    dw.close()


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [METHOD, METHOD | po.OR_F_BEAM, po.OR_F_L4])
@pytest.mark.parametrize("pose", [((256.0, 140.0, 256.0), 0.0, -15.0),
                                  ((180.5, 108.25, 330.75), 2.3, -40.0),
                                  ((300.0, 100.0, 100.0), 4.0, -65.0)])
def test_device_ao_equals_oracle_c1(c1, c1_oracle_world, flags, pose):
    vg, dw = c1
    pos, yaw, pitch = pose
    cam = vg.camera_from_pose(pos, yaw, math.radians(pitch), math.radians(70.0), 333, 187)
    cam.jitter_x, cam.jitter_y = 0.25, -0.375
    p = vg.default_params(flags)
    rec, _ = vg.render_primary(dw, cam, p)
    ao = vg.render_ao(dw, cam, rec).cpu().numpy()
    r = vg.records(rec)
    want = po.render_ao(c1_oracle_world, cam, r)
    assert np.array_equal(ao.view(np.uint32), want.view(np.uint32))
    if pose[2] <= -40.0:
        assert (ao < 1.0).mean() > 0.05


@pytest.mark.gpu
def test_device_ao_shifted_window():
    import voxelg_b200 as vg
    w, wo, _ = scenes.floor_pillars(origin_chunk=(3, 5))
    w.rebuild()
    dw = vg.DeviceWorld(*scenes.DEFAULT_BRICKS)
    dw.upload(w.a)
    cam = vg.camera_from_pose((wo[0] + 36.0, 95.0, wo[2] + 30.0), 0.7, math.radians(-50.0),
                              math.radians(70.0), 256, 144, world_origin=wo)
    rec, _ = vg.render_primary(dw, cam, vg.default_params(METHOD))
    ao = vg.render_ao(dw, cam, rec).cpu().numpy()
    want = po.render_ao(w, cam, vg.records(rec))
    assert np.array_equal(ao.view(np.uint32), want.view(np.uint32))
    assert (ao < 1.0).any()
    dw.close()


@pytest.mark.gpu
def test_device_ao_c2_full_frame():
    """The full benchmark frame (2048x256x2048, 1920x1080, beam/LUT/LOD/shadow)."""
    import voxelg_b200 as vg
    cfg = vg.CONFIGS["c2"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    cam = vg.default_camera(dw, cfg.width, cfg.height)
    rec, _ = vg.render_primary(dw, cam, vg.default_params(cfg.flags))
    ao = vg.render_ao(dw, cam, rec).cpu().numpy()
    arrays = dw.download()
    ow = po.World(*cfg.bricks, arrays=arrays)
    want = po.render_ao(ow, cam, vg.records(rec))
    assert np.array_equal(ao.view(np.uint32), want.view(np.uint32))
    dw.close()
