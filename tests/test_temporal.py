"""Temporal-differential tile gating: project_brick_to_tiles
(src/temporal.rs:16-111), the rotating refresh (src/app.rs:706-725) and the
cs_main tile gate (shaders/raymarch.wgsl:580-587)."""
import math

import numpy as np
import pytest

from oracle import pyoracle as po

W, H = 320, 180


def camera(world_origin=(0, 0, 0)):
    return po.camera_from_pose((256.0 + world_origin[0], 140.0, 256.0 + world_origin[2]), 0.4,
                               math.radians(-15.0), math.radians(70.0), W, H, world_origin)


def bits(mask, n):
    return np.array([(mask[i >> 5] >> (i & 31)) & 1 for i in range(n)], bool)


def test_projection_marks_visible_brick_only():
    w = po.World(128, 64, 128)
    cam = camera()
    n_tiles = ((W + 7) // 8) * ((H + 7) // 8)
    # a brick well in front of the camera covers a few tiles
    fwd = np.array(list(cam.forward))
    p = np.array([256.0, 140.0, 256.0]) + 60 * fwd
    bi = int(p[0] // 4) + int(p[1] // 4) * 128 + int(p[2] // 4) * 128 * 64
    m = bits(po.project_dirty(w, cam, [bi]), n_tiles)
    assert 0 < m.sum() < 40
    # a brick straddling the camera plane marks the whole screen
    bi = 64 + 35 * 128 + 64 * 128 * 64
    m = bits(po.project_dirty(w, cam, [bi]), n_tiles)
    assert m.all()
    # a brick behind the camera marks nothing
    p = np.array([256.0, 140.0, 256.0]) - 40 * fwd
    bi = int(p[0] // 4) + int(p[1] // 4) * 128 + int(p[2] // 4) * 128 * 64
    assert not bits(po.project_dirty(w, cam, [bi]), n_tiles).any()


def test_refresh_rotation_covers_every_tile_once():
    n_tiles = ((W + 7) // 8) * ((H + 7) // 8)
    spread = 8
    counts = np.zeros(n_tiles, int)
    for phase in range(spread):
        m = po.refresh_tiles(W, H, spread, phase, np.zeros((n_tiles + 31) // 32, np.uint32))
        counts += bits(m, n_tiles)
    assert (counts == 1).all()


@pytest.fixture(scope="module")
def vg_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200
    return voxelg_b200


@pytest.mark.gpu
@pytest.mark.parametrize("origin_chunk", [(0, 0), (3, 5)])
def test_device_projection_matches_oracle(vg_gpu, c1_oracle_world, origin_chunk):
    import torch
    vg = vg_gpu
    ro = (origin_chunk[0] * 32, 0, origin_chunk[1] * 32)
    dw = vg.DeviceWorld(128, 64, 128)
    vcam = vg.camera_from_pose((256.0 + ro[0], 140.0, 256.0 + ro[2]), 0.4, math.radians(-15.0),
                               math.radians(70.0), W, H, ro)
    rng = np.random.default_rng(4)
    idx = rng.integers(0, 128 * 64 * 128, 3000).astype(np.uint32)
    nw = vg.tile_mask_words(W, H)
    mask = torch.zeros(nw, dtype=torch.int32, device="cuda")
    vg.project_dirty(dw, vcam, idx, mask)
    want = po.project_dirty(c1_oracle_world, vcam, idx)
    assert np.array_equal(mask.cpu().numpy().view(np.uint32), want)
    assert 0 < np.unpackbits(want.view(np.uint8)).sum()
    # refresh rotation
    for spread, phase in ((8, 3), (4, 0)):
        mask.zero_()
        vg.tile_refresh(W, H, spread, phase, mask)
        want = po.refresh_tiles(W, H, spread, phase, np.zeros(nw, np.uint32))
        assert np.array_equal(mask.cpu().numpy().view(np.uint32), want)
    dw.close()


@pytest.mark.gpu
def test_gated_frame_retraces_dirty_tiles_only(vg_gpu, c1_oracle_world):
    """Edit the world, project the dirty bricks, re-trace only those tiles:
    dirty tiles equal a full frame of the edited world, clean tiles keep the
    previous frame."""
    import torch
    vg = vg_gpu
    src = c1_oracle_world
    hw = vg.HostWorld(*src.dims)
    for k in po.World.NAMES:
        hw.arrays[k][...] = src.a[k].view(hw.arrays[k].dtype)
    hw.rebuild()
    dw = vg.DeviceWorld(*src.dims)
    dw.sync(hw)
    cam = vg.default_camera(dw, W, H)
    p = vg.default_params()
    rec0, sh0 = vg.render_primary(dw, cam, p)
    prev_rec, prev_sh = rec0.clone(), sh0.clone()
    # a crater and a tower in view
    for x in range(240, 272):
        for z in range(300, 332):
            for y in range(60, 140):
                hw.set_voxel(x, y, z, 0 if y < 110 else 4)
    dirty_idx = np.array(sorted({(x // 4) + (y // 4) * 128 + (z // 4) * 128 * 64
                                 for x in range(240, 272) for z in range(300, 332)
                                 for y in range(60, 140)}), np.uint32)
    dw.sync(hw)
    mask = torch.zeros(vg.tile_mask_words(W, H), dtype=torch.int32, device="cuda")
    vg.project_dirty(dw, cam, dirty_idx, mask)
    rec, sh = prev_rec.clone(), prev_sh.clone()
    vg.render_primary_gated(dw, cam, p, mask, rec, sh)
    full_rec, full_sh = vg.render_primary(dw, cam, p)
    torch.cuda.synchronize()
    m = mask.cpu().numpy().view(np.uint32)
    tw = (W + 7) // 8
    tile_of = ((np.arange(H)[:, None] // 8) * tw + np.arange(W)[None, :] // 8).reshape(-1)
    dirty_px = ((m[tile_of >> 5] >> (tile_of & 31)) & 1).astype(bool)
    assert 0 < dirty_px.sum() < len(dirty_px)
    r, fr, pr = (vg.records(x).view(np.uint8).reshape(-1, 24) for x in (rec, full_rec, prev_rec))
    assert np.array_equal(r[dirty_px], fr[dirty_px])
    assert np.array_equal(r[~dirty_px], pr[~dirty_px])
    assert not np.array_equal(fr[dirty_px], pr[dirty_px]), "the edit changed nothing visible"
    s, fs, ps = (vg.shadows(x).view(np.uint8).reshape(-1, 8) for x in (sh, full_sh, prev_sh))
    assert np.array_equal(s[dirty_px], fs[dirty_px]) and np.array_equal(s[~dirty_px], ps[~dirty_px])
    dw.close()
    hw.close()
