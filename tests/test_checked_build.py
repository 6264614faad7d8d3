"""The checked library (libvoxrt_checked.so): every world-array load of the
traversal is compared with the array's length first, and the first bad index
is kept in a per-world word (vx_world_oob).  With no memory checker available,
it stands in for one: the traversal workloads of the parity tests run on it
with no bad index recorded and records still equal to the oracle's.

Run as a script (the GPU test does so, in a child process with
VOXRT_CHECKED=1), this file runs those workloads."""
import ctypes as C
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle as po  # noqa: E402

LIBDIR = ROOT / "voxelg_b200" / "lib"


def declared_symbols():
    text = (ROOT / "include" / "voxrt.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vx_\w+)\s*\(", text)))


def test_checked_library_exports_the_abi_and_says_so():
    plain = C.CDLL(str(LIBDIR / "libvoxrt.so"))
    checked = C.CDLL(str(LIBDIR / "libvoxrt_checked.so"))
    for name in declared_symbols():
        getattr(checked, name)
    assert plain.vx_checked_build() == 0
    assert checked.vx_checked_build() == 1


def _workloads():
    """Every traversal kernel on the checked library, each compared with the
    oracle and followed by a read of the world's bad-index word."""
    import torch

    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    from voxelg_b200 import learned as vl
    from voxelg_b200 import queue as q
    assert L.load().vx_checked_build() == 1, "VOXRT_CHECKED=1 must load the checked library"
    flags = po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    ow = po.World(*cfg.bricks)
    ow.generate(cfg.terrain)
    done = []

    def clean(what):
        torch.cuda.synchronize()
        word = dw.oob()
        assert word == 0, f"{what}: array {word >> 56}, index {word & ((1 << 56) - 1)}"
        done.append(what)

    def same(got, want, what):
        assert np.array_equal(np.ascontiguousarray(got).view(np.uint8),
                              np.ascontiguousarray(want).view(np.uint8)), what

    # frames: grid and persistent schedules, two flag sets, camera inside and above
    for pose in [((256.0, 140.0, 256.0), 0.0, -0.26), ((100.5, 97.3, 410.2), 2.1, -0.6)]:
        cam = vg.camera_from_pose(pose[0], pose[1], pose[2], 1.2, 160, 90)
        for fl in (flags | po.OR_F_SHADOW, po.OR_F_L4):
            p = vg.default_params(fl)
            want, wsh, _, _, _ = po.render_frame(ow, cam, p)
            for persistent in (False, True):
                dw.set_persistent(persistent)
                rec, sh = vg.render_primary(dw, cam, p)
                same(vg.records(rec), want, "frame")
                if sh is not None:
                    same(vg.shadows(sh), wsh, "shadow")
                clean(f"frame persistent={persistent} flags={fl}")
            dw.set_persistent(False)
            if fl & po.OR_F_SHADOW:
                ao = vg.render_ao(dw, cam, rec).cpu().numpy()
                same(ao, po.render_ao(ow, cam, want), "ao")
                clean("ao")
    # generic rays of the three kinds, from inside, outside and degenerate
    rng = np.random.default_rng(3)
    n = 6000
    rays = np.zeros(n, po.RAY)
    rays["org"] = rng.uniform([-60, -20, -60], [572, 300, 572], (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[::17] = 0.0
    d[1::23] *= np.float32(1e-20)
    rays["dir"] = d
    rays["tmax"] = rng.uniform(1, 800, n).astype(np.float32)
    for kind in (0, 1, 2):
        rays["kind"] = kind
        p = vg.default_params(flags)
        same(vg.records(vg.trace(dw, rays, p)), po.trace_batch(ow, rays, p)[0], f"kind {kind}")
        clean(f"trace kind {kind}")
    # picking: batch and single calls
    picks, hits = vg.raycast_batch(dw, rays["org"], d)
    wpicks, whits, _ = po.raycast_batch(ow, rays["org"], d)
    same(hits, whits, "pick hits")
    same(picks, wpicks, "picks")
    for i in range(0, 40, 4):
        h = vg.raycast(rays["org"][i], d[i], dw)
        assert (h is not None) == bool(whits[i])
    clean("raycast")
    # the mixed queue, sorted and not
    cam = vg.default_camera(dw, 160, 90)
    qrays, _ = q.mixed_queue(cfg.bricks, cam, 160, 90, 5, probe_radius=48, pick_rays=2000)
    p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_SHADOW)
    want, wsh, _, _ = po.trace_batch(ow, qrays, p, shadows=True)
    for so in (0, 1):
        t = q.default_tuning()
        t.block_threads, t.refill_min, t.sort = 256, 32, so
        _, out, sh = q.run(dw, qrays, p, tuning=t)
        same(out.cpu().numpy(), want, f"queue sort={so}")
        same(sh.cpu().numpy(), wsh, f"queue shadows sort={so}")
        clean(f"queue sort={so}")
    # the learned form's verification walk and restart (no network)
    p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD)
    plain, _ = vg.render_primary(dw, cam, p)
    rec = torch.empty_like(plain)
    vl.render_learned(dw, None, cam, p, rec)
    a, b = vg.records(plain).copy(), vg.records(rec).copy()
    a["steps"] = 0
    b["steps"] = 0
    same(a, b, "learned")
    clean("learned")
    # the device-resident request loop over the generic rays (degenerate ones included)
    import voxelg_b200.serve as sv
    p = vg.default_params(flags)
    srv = sv.Server(dw, p, mem_budget_bytes=8 << 20, resident=True)
    try:
        for kind in (0, 1, 2):
            rays["kind"] = kind
            same(srv.wait(srv.submit(rays)), po.trace_batch(ow, rays, p)[0],
                 f"resident kind {kind}")
    finally:
        srv.close()
    clean("resident request loop")
    # a streamed window with edits (generator, edit replay, per-tile words)
    dw.fill_window(0xC0FFEE_F00D_BEEF, 0, 0)
    dw.apply_edit(300, 90, 200, 18)
    dw.shift_origin(3, -2)
    sw = po.World(*cfg.bricks)
    po.fill_window(sw, 0xC0FFEE_F00D_BEEF, 3, -2)
    wo = (96, 0, -64)
    sw.set_voxel(300 % 512, 90, 200 % 512, 18)   # slot of world voxel (300, 90, 200)
    cam = vg.camera_from_pose((wo[0] + 256.0, 150.0, wo[2] + 256.0), 0.5, -0.4, 1.2, 128, 72,
                              world_origin=wo)
    p = vg.default_params(flags | po.OR_F_SHADOW)
    same(vg.records(vg.render_primary(dw, cam, p)[0]), po.render_frame(sw, cam, p)[0],
         "streamed window")
    clean("streamed window")
    dw.close()
    return done


@pytest.mark.gpu
def test_checked_library_runs_the_parity_workloads_clean():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    env = dict(os.environ, VOXRT_CHECKED="1")
    r = subprocess.run([sys.executable, str(Path(__file__).resolve())], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "checked workloads clean: 19" in r.stdout, r.stdout[-2000:]


if __name__ == "__main__":
    ran = _workloads()
    print(f"checked workloads clean: {len(ran)}")
