"""vx_render_primary_noalloc: the primary frame for callers that cannot call
cudaMalloc.

Such a caller is a host that reserves all of its device memory up front and
hands plugins pre-allocated buffers (an engine frame loop, a sandboxed plugin
host): it owns the world in device memory and the output records, and a
device allocation mid-frame is either forbidden or a stall.  This test plays
that caller: every device buffer is allocated up front with torch, the world
is laid out in the library's device layout, and the entry point is called
through the C ABI twice in a row, with two different cameras, each output
checked bit for bit against the allocating entry point vx_render_primary.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def test_noalloc_matches_render_primary_twice():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    view, keep = caller_owned_world(torch, dw.download(), cfg.bricks, device)

    import math
    cams = [vg.default_camera(dw, 640, 360),
            vg.camera_from_pose((40.0, 170.0, 480.0), 2.3, -0.45, math.radians(70), 640, 360)]
    p = vg.default_params()  # beam + LUT + LOD + shadow: the beam scratch is used
    n = 640 * 360
    outs = [(torch.empty(n * 24, dtype=torch.uint8, device=device),
             torch.empty(n * 8, dtype=torch.uint8, device=device)) for _ in cams]
    torch.cuda.synchronize()
    lib = L.load()
    free_before = None
    for i, (cam, (rec, sh)) in enumerate(zip(cams, outs)):
        if i == 1:
            free_before = torch.cuda.mem_get_info(device)[0]
        rc = lib.vx_render_primary_noalloc(C.byref(view), C.byref(cam), C.byref(p),
                                           C.c_void_p(rec.data_ptr()), C.c_void_p(sh.data_ptr()),
                                           C.c_void_p(0))
        assert rc == 0, lib.vx_last_error()
        torch.cuda.synchronize()
        if i == 1:
            assert torch.cuda.mem_get_info(device)[0] == free_before, "device memory changed"
        want_rec, want_sh = vg.render_primary(dw, cam, p)
        torch.cuda.synchronize()
        assert torch.equal(rec, want_rec), f"call {i}: records differ from vx_render_primary"
        assert torch.equal(sh, want_sh), f"call {i}: shadow records differ"
        assert (vg.records(rec)["flags"] & 1).any()
    assert not torch.equal(outs[0][0], outs[1][0])
    dw.close()


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
