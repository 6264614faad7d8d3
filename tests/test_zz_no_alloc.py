"""vx_render_primary_noalloc: the primary frame for callers that cannot call
cudaMalloc.

Such a caller is a host that reserves all of its device memory up front and
hands plugins pre-allocated buffers (an engine frame loop, a sandboxed plugin
host): it owns the world in device memory and the output records, and a
device allocation mid-frame is either forbidden or a stall.  These tests play
that caller: every device buffer is allocated up front with torch, the world
is laid out in the library's device layout, and the entry point is called
through the C ABI.

- Two calls in a row (two cameras), with and without the beam pre-pass (the
  one user of the static scratch), on the legacy default stream and on a
  caller-owned stream: each output equals the allocating entry point
  vx_render_primary bit for bit, and no call after the first changes the
  device's free memory.
- The walk of a caller-owned world tests the L4, chunk and tile masks
  directly (it has no per-tile skip word), so its frames are also checked
  against the oracle on extreme worlds (all solid, 3D checkerboard, sparse
  voxels of every material class) and on seeded random worlds with random
  window origins.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from scenes import pattern_world, random_world

pytestmark = pytest.mark.gpu

METHOD = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM


def caller_owned_world(torch, host, dims, device):
    """Device copies, owned by the caller, of a world's arrays."""
    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device)
    t = {
        "occupancy": dev(host["bricks"]["occupancy"].view(np.int64)),
        "materials": dev(host["bricks"]["materials"].reshape(-1)),
        "tile_mask": dev(host["tile_mask"].view(np.int64)),
        "chunk_mask": dev(host["chunk_mask"].view(np.int64)),
        "l4_mask": dev(host["l4_mask"].view(np.int64)),
        "brick_uniform": dev(host["brick_uniform"]),
        "tile_uniform": dev(host["tile_uniform"]),
    }
    from voxelg_b200 import _lib as L
    view = L.VxWorldView(dims[0], dims[1], dims[2], *[t[k].data_ptr() for k in
                         ("occupancy", "materials", "tile_mask", "chunk_mask", "l4_mask",
                          "brick_uniform", "tile_uniform")])
    return view, t


def noalloc_frame(torch, lib, view, cam, p, device, stream=None):
    """One call through the C ABI into caller-owned record buffers."""
    n = int(cam.res_x) * int(cam.res_y)
    rec = torch.empty(n * 24, dtype=torch.uint8, device=device)
    sh = torch.empty(n * 8, dtype=torch.uint8, device=device)
    torch.cuda.synchronize()
    handle = C.c_void_p(stream.cuda_stream if stream is not None else 0)
    rc = lib.vx_render_primary_noalloc(C.byref(view), C.byref(cam), C.byref(p),
                                       C.c_void_p(rec.data_ptr()), C.c_void_p(sh.data_ptr()),
                                       handle)
    assert rc == 0, lib.vx_last_error()
    torch.cuda.synchronize()
    return rec, sh


@pytest.mark.parametrize("beam", [True, False], ids=["beam", "no_beam"])
@pytest.mark.parametrize("own_stream", [False, True], ids=["null_stream", "caller_stream"])
def test_noalloc_matches_render_primary_twice(beam, own_stream):
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import math

    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    view, keep = caller_owned_world(torch, dw.download(), cfg.bricks, device)
    cams = [vg.default_camera(dw, 640, 360),
            vg.camera_from_pose((40.0, 170.0, 480.0), 2.3, -0.45, math.radians(70), 640, 360)]
    flags = METHOD | po.OR_F_SHADOW
    if not beam:
        flags &= ~po.OR_F_BEAM
    p = vg.default_params(flags)
    stream = torch.cuda.Stream(device) if own_stream else None
    lib = L.load()
    outs = []
    for i, cam in enumerate(cams):
        n = int(cam.res_x) * int(cam.res_y)
        rec = torch.empty(n * 24, dtype=torch.uint8, device=device)
        sh = torch.empty(n * 8, dtype=torch.uint8, device=device)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(device)[0]
        handle = C.c_void_p(stream.cuda_stream if stream is not None else 0)
        rc = lib.vx_render_primary_noalloc(C.byref(view), C.byref(cam), C.byref(p),
                                           C.c_void_p(rec.data_ptr()), C.c_void_p(sh.data_ptr()),
                                           handle)
        assert rc == 0, lib.vx_last_error()
        torch.cuda.synchronize()
        if i == 1:
            # the first call of the process may load the module (and its
            # static array); later calls must leave free memory unchanged
            assert torch.cuda.mem_get_info(device)[0] == free_before, "device memory changed"
        want_rec, want_sh = vg.render_primary(dw, cam, p)
        torch.cuda.synchronize()
        assert torch.equal(rec, want_rec), f"call {i}: records differ from vx_render_primary"
        assert torch.equal(sh, want_sh), f"call {i}: shadow records differ"
        assert (vg.records(rec)["flags"] & 1).any()
        outs.append(rec)
    assert not torch.equal(outs[0], outs[1])
    dw.close()


def _check_against_oracle(torch, lib, ow, cams, flag_sets, device):
    import voxelg_b200 as vg
    view, keep = caller_owned_world(torch, ow.a, ow.dims, device)
    for cam in cams:
        for flags in flag_sets:
            p = vg.default_params(flags)
            rec, sh = noalloc_frame(torch, lib, view, cam, p, device)
            wrec, wsh, _, _, _ = po.render_frame(ow, cam, p)
            got = rec.cpu().numpy()
            bad = np.flatnonzero((got.reshape(-1, 24) != wrec.view(np.uint8).reshape(-1, 24))
                                 .any(axis=1))
            assert bad.size == 0, f"flags={flags}: {bad.size} records differ, first {bad[:5]}"
            if flags & po.OR_F_SHADOW:
                assert np.array_equal(sh.cpu().numpy(), wsh.view(np.uint8)), f"flags={flags}"


@pytest.mark.parametrize("kind", ["full", "checker", "sparse"])
def test_noalloc_pattern_worlds_match_oracle(kind):
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    ow = pattern_world(kind)
    cams = [vg.camera_from_pose(pose[0], pose[1], pose[2], 1.2, 96, 54)
            for pose in [((128.5, 30.2, 128.5), 0.4, -0.3), ((3.0, 63.0, 250.0), 2.2, -0.9)]]
    _check_against_oracle(torch, L.load(), ow, cams,
                          (METHOD | po.OR_F_SHADOW, po.OR_F_L4, po.OR_F_LUT | po.OR_F_LOD),
                          device)


@pytest.mark.parametrize("seed", range(6))
def test_noalloc_random_worlds_match_oracle(seed):
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    rng = np.random.default_rng(5000 + seed)
    ow = random_world(rng)
    VX, VY, VZ = ow.voxels
    wo = (int(rng.integers(-3, 4)) * 32 + int(rng.integers(0, 32)), 0,
          int(rng.integers(-3, 4)) * 32 + int(rng.integers(0, 32)))
    cams = []
    for _ in range(2):
        pos = (wo[0] + float(rng.uniform(-20, VX + 20)), float(rng.uniform(5, 120)),
               wo[2] + float(rng.uniform(-20, VZ + 20)))
        cams.append(vg.camera_from_pose(pos, float(rng.uniform(0, 6.28)),
                                        float(rng.uniform(-1.2, 0.6)), 1.2, 80, 45,
                                        world_origin=wo))
    _check_against_oracle(torch, L.load(), ow, cams,
                          (METHOD | po.OR_F_SHADOW, po.OR_F_LOD | po.OR_F_SHADOW, 0), device)


def test_noalloc_rejects_frames_beyond_the_scratch():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    lib = L.load()
    view = L.VxWorldView(128, 64, 128, 256, 256, 256, 256, 256, 256, 256)
    cam = vg.camera_from_pose((256.0, 140.0, 256.0), 0.0, -0.26, 1.22, 4096, 2304)
    p = vg.default_params()
    rc = lib.vx_render_primary_noalloc(C.byref(view), C.byref(cam), C.byref(p),
                                       C.c_void_p(256), C.c_void_p(0), C.c_void_p(0))
    assert rc == L.VX_ERR_INVALID
    assert b"static beam scratch" in lib.vx_last_error()
