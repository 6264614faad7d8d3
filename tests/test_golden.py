"""Known-answer vectors (tests/golden/traversal.json) against the oracle and
every traversal entry point.

The vectors come from tests/golden/make_golden.py, an exact binary32
emulation of the reference's WGSL traversal and CPU picking walk over worlds
described as boxes, cross-checked by exact ray/box geometry and by records
worked out by hand.  It shares no code with the C oracle or the kernels.
The worlds' arrays are built here from the boxes with numpy (a third
builder of the masks and uniform bytes, checked against the oracle's).

Pinned: first-hit (trace), any-hit (trace_any) and no-water rays with their
distance caps and iteration caps; the L4 / chunk / tile / brick skips and
skip_to_cell's landing; uniform tile and brick exits; brick LOD beyond 400
(topmost material, recorded at the voxel where the walk stands) and tile
LOD beyond 520 (representative material); the 700 distance budget; glass,
far water, far leaves, decoration and turf; toroidal slots of a window whose
origin is not cell aligned; camera rays through ray_dir_uv; the beam
pre-pass (beam.wgsl: the block-centre ray's tile walk in world coordinates,
its skip of the pixel rays' origins, t re-based); picking.
"""
import ctypes as C
import importlib.util
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "traversal.json")
GOLDEN = json.load(open(FIXTURE))
WORLDS = {w["name"]: w for w in GOLDEN["worlds"]}


# ------------------------------------------------------------ world arrays


def slot_voxels(w):
    """Materials in slot space, indexed [z, y, x]."""
    bx, by, bz = w["bricks"]
    V = (4 * bx, 4 * by, 4 * bz)
    ro = w["origin"]
    vox = np.zeros((V[2], V[1], V[0]), np.uint8)
    for x0, y0, z0, x1, y1, z1, m in w["boxes"]:
        xs = [(x - ro[0]) for x in range(x0, x1)]
        zs = [(z - ro[2]) for z in range(z0, z1)]
        sx = np.array([(x + ro[0]) % V[0] for x in xs])
        sz = np.array([(z + ro[2]) % V[2] for z in zs])
        vox[np.ix_(sz, np.arange(y0, y1), sx)] = m
    return vox


def _pack_children(nonempty, n4):
    """Parent words from a [z, y, x] child grid: bit lx + 4 lz + 16 ly."""
    pz, py, px = n4
    g = np.zeros((pz * 4, py * 4, px * 4), bool)
    g[:nonempty.shape[0], :nonempty.shape[1], :nonempty.shape[2]] = nonempty
    b = g.reshape(pz, 4, py, 4, px, 4).transpose(0, 2, 4, 3, 1, 5).reshape(-1, 64)
    return np.packbits(b, axis=1, bitorder="little").view("<u8").reshape(-1)


def world_arrays(w):
    """The host layout (bricks, tile / chunk / L4 masks, uniform bytes)."""
    bx, by, bz = w["bricks"]
    vox = slot_voxels(w)
    mats = vox.reshape(bz, 4, by, 4, bx, 4).transpose(0, 2, 4, 3, 1, 5).reshape(-1, 64)
    bricks = np.zeros(len(mats), po.BRICK)
    bricks["materials"] = mats
    bricks["occupancy"] = np.packbits(mats != 0, axis=1, bitorder="little").view("<u8")[:, 0]
    nonempty = (mats != 0).any(axis=1).reshape(bz, by, bx)
    tx, ty, tz = bx // 4, by // 4, bz // 4
    cx, cy, cz = (tx + 3) // 4, (ty + 3) // 4, (tz + 3) // 4
    lx, ly, lz = (cx + 3) // 4, (cy + 3) // 4, (cz + 3) // 4
    tile_mask = _pack_children(nonempty, (tz, ty, tx))
    tile_ne = (tile_mask != 0).reshape(tz, ty, tx)
    chunk_mask = _pack_children(tile_ne, (cz, cy, cx))
    chunk_ne = (chunk_mask != 0).reshape(cz, cy, cx)
    l4_mask = _pack_children(chunk_ne, (lz, ly, lx))
    full = (mats != 0).all(axis=1) & (mats == mats[:, :1]).all(axis=1)
    bu = np.where(full, mats[:, 0], 0).astype(np.uint8)
    b3 = bu.reshape(tz, 4, ty, 4, tx, 4).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 64)
    tu = np.where((b3 != 0).all(axis=1) & (b3 == b3[:, :1]).all(axis=1), b3[:, 0], 0)
    return {"bricks": bricks, "tile_mask": tile_mask, "chunk_mask": chunk_mask,
            "l4_mask": l4_mask, "brick_uniform": bu, "tile_uniform": tu.astype(np.uint8)}


_ORACLE_WORLDS = {}


def oracle_world(name):
    if name not in _ORACLE_WORLDS:
        w = WORLDS[name]
        _ORACLE_WORLDS[name] = po.World(*w["bricks"], arrays=world_arrays(w))
    return _ORACLE_WORLDS[name]


# ------------------------------------------------------------ cases


def params_of(pj, product=False):
    if product:
        import voxelg_b200 as vg
        p = vg.default_params(pj["flags"])
    else:
        p = po.default_params(pj["flags"])
    p.max_dist, p.lod_brick_t, p.tile_lod_t = pj["max_dist"], pj["lod_brick_t"], pj["tile_lod_t"]
    p.max_iters, p.any_max_iters = pj["max_iters"], pj["any_max_iters"]
    return p


def ray_groups():
    """Rays grouped by (world, params): [(world, params json, rays, expected)]."""
    groups = {}
    for r in GOLDEN["rays"]:
        key = (r["world"], json.dumps(r["params"], sort_keys=True))
        groups.setdefault(key, []).append(r)
    out = []
    for (name, pj), rs in sorted(groups.items()):
        rays = np.zeros(len(rs), po.RAY)
        rays["org"] = [r["org"] for r in rs]
        rays["dir"] = [r["dir"] for r in rs]
        rays["tmax"] = [r["tmax"] for r in rs]
        rays["kind"] = [r["kind"] for r in rs]
        out.append((name, json.loads(pj), rays, rs))
    return out


def expected_records(exps):
    e = np.zeros(len(exps), po.RECORD)
    for i, x in enumerate(exps):
        if x is None:
            continue
        e[i]["voxel"] = x["voxel"]
        e[i]["face"], e[i]["mat"], e[i]["flags"] = x["face"], x["mat"], x["flags"]
        e[i]["t"] = np.float32(x["t"])
        e[i]["steps"] = x["steps"]
    return e


def assert_records(got, exps, what, steps=True, cases=None):
    got = np.ascontiguousarray(got).view(po.RECORD)
    want = expected_records(exps)
    live = np.array([x is not None for x in exps])
    bad = []
    for f in ("voxel", "face", "mat", "flags", "t", "steps"):
        if f == "steps" and not steps:
            continue
        a, b = got[f], want[f]
        if f == "t":
            a, b = a.view(np.uint32), b.view(np.uint32)
        diff = (a != b) if a.ndim == 1 else (a != b).any(axis=1)
        bad.extend(np.flatnonzero(diff & live).tolist())
    bad = sorted(set(bad))
    if bad:
        i = bad[0]
        why = cases[i].get("why") if cases else ""
        raise AssertionError(f"{what}: {len(bad)} of {int(live.sum())} records differ; "
                             f"first #{i} ({why}): got {got[i]}, want {want[i]}")


def camera_of(cj, product=False):
    if product:
        from voxelg_b200 import _lib as L
        c = L.VxCamera()
    else:
        c = po.OrCamera()
    for k in ("origin", "forward", "right", "up"):
        for i in range(3):
            getattr(c, k)[i] = cj[k][i]
    c.tan_half_fov = cj["tan_half_fov"]
    c.res_x, c.res_y = float(cj["res"][0]), float(cj["res"][1])
    c.jitter_x, c.jitter_y = cj["jitter"]
    for i in range(3):
        c.world_origin[i] = cj["world_origin"][i]
    return c


# ------------------------------------------------------------ CPU


def test_fixture_is_what_the_generator_computes():
    """The committed vectors are the committed generator's output."""
    spec = importlib.util.spec_from_file_location("make_golden",
                                                  os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    fresh = json.loads(json.dumps(mg.build()))
    assert fresh == GOLDEN


def test_fixture_covers_the_pinned_behaviour():
    why = {}
    for r in GOLDEN["rays"]:
        why[r["why"]] = why.get(r["why"], 0) + 1
    for k in ("hand", "voxel", "uniform tile", "uniform brick", "brick LOD", "tile LOD", "miss"):
        assert why.get(k, 0) > 0, (k, why)
    kinds = {r["kind"] for r in GOLDEN["rays"]}
    assert kinds == {0, 1, 2}
    ts = [r["expect"]["t"] for r in GOLDEN["rays"] if r["expect"]["flags"] & 1]
    for lo, hi in ((399, 400), (400, 401), (519, 520), (520, 521), (699, 700)):
        assert any(lo <= t <= hi for t in ts), (lo, hi)
    assert any(r["expect"]["steps"] == r["params"]["max_iters"] for r in GOLDEN["rays"])
    assert any(p["expect"] is None for p in GOLDEN["picks"])
    assert any(p["expect"] is not None for p in GOLDEN["picks"])


@pytest.mark.parametrize("name", sorted(WORLDS))
def test_world_builder_matches_oracle_rebuild(name):
    """The numpy builder above and the oracle's mask / uniform rebuild agree."""
    w = WORLDS[name]
    a = world_arrays(w)
    ow = po.World(*w["bricks"], arrays={k: v.copy() for k, v in a.items()})
    for k in ("tile_mask", "chunk_mask", "l4_mask", "brick_uniform", "tile_uniform"):
        ow.a[k][:] = 0
    ow.rebuild()
    for k in ("tile_mask", "chunk_mask", "l4_mask", "brick_uniform", "tile_uniform"):
        assert np.array_equal(ow.a[k], a[k]), k


def test_oracle_rays_match_golden():
    for name, pj, rays, cases in ray_groups():
        out, _, _ = po.trace_batch(oracle_world(name), rays, params_of(pj),
                                   origin=WORLDS[name]["origin"], threads=4)
        assert_records(out, [c["expect"] for c in cases], f"oracle {name} {pj}", cases=cases)


def test_oracle_frames_match_golden():
    for fr in GOLDEN["frames"]:
        rec, _, beam, _, _ = po.render_frame(oracle_world(fr["world"]), camera_of(fr["camera"]),
                                             params_of(fr["params"]), threads=4)
        assert_records(rec, fr["expect"], f"oracle frame {fr['world']} {fr['params']['flags']}")
        if fr["params"]["flags"] & 8:
            # the beam pre-pass itself (beam.wgsl): one first-tile t per 8x8 block
            want = np.array(fr["beam"], np.float32).reshape(-1)
            assert np.array_equal(beam.view(np.uint32), want.view(np.uint32)), fr["world"]


def test_oracle_picks_match_golden():
    for pk in GOLDEN["picks"]:
        hit, vox, nrm, _ = po.raycast(oracle_world(pk["world"]), pk["cam"], pk["dir"],
                                      origin=WORLDS[pk["world"]]["origin"])
        e = pk["expect"]
        assert hit == (e is not None), pk
        if e is not None:
            assert list(vox) == e["voxel"] and list(nrm) == e["normal"], (pk, vox, nrm)


# ------------------------------------------------------------ GPU


@pytest.fixture(scope="module")
def device_worlds():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    out = {}
    for name, w in WORLDS.items():
        dw = vg.DeviceWorld(*w["bricks"])
        dw.upload(world_arrays(w))
        out[name] = dw
    yield out
    for dw in out.values():
        dw.close()


@pytest.mark.gpu
def test_trace_kernel_matches_golden(device_worlds):
    import voxelg_b200 as vg
    for name, pj, rays, cases in ray_groups():
        out = vg.trace(device_worlds[name], rays, params_of(pj, True),
                       origin=WORLDS[name]["origin"])
        assert_records(vg.records(out), [c["expect"] for c in cases], f"vx_trace {name} {pj}",
                       cases=cases)


@pytest.mark.gpu
def test_queue_matches_golden(device_worlds):
    import torch
    from voxelg_b200 import queue as vq
    for sort in (0, 1):
        for name, pj, rays, cases in ray_groups():
            tun = vq.default_tuning()
            tun.sort = sort
            _, out, _ = vq.run(device_worlds[name], rays, params_of(pj, True), tuning=tun,
                               origin=WORLDS[name]["origin"], with_shadow=False)
            torch.cuda.synchronize()
            assert_records(out.cpu().numpy(), [c["expect"] for c in cases],
                           f"queue sort={sort} {name} {pj}", cases=cases)


@pytest.mark.gpu
def test_frames_match_golden(device_worlds):
    """The frame kernel (per-CTA and persistent schedules) and the
    no-allocation entry point, per golden camera."""
    import torch
    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    from test_zz_no_alloc import caller_owned_world
    for fr in GOLDEN["frames"]:
        dw = device_worlds[fr["world"]]
        cam, p = camera_of(fr["camera"], True), params_of(fr["params"], True)
        for persistent in (False, True):
            dw.set_persistent(persistent)
            rec, _ = vg.render_primary(dw, cam, p)
            torch.cuda.synchronize()
            assert_records(vg.records(rec), fr["expect"],
                           f"frame persistent={persistent} {fr['world']} {fr['params']['flags']}")
        dw.set_persistent(False)
        view, keep = caller_owned_world(torch, world_arrays(WORLDS[fr["world"]]),
                                        WORLDS[fr["world"]]["bricks"], torch.device("cuda", 0))
        n = int(cam.res_x) * int(cam.res_y)
        rec = torch.empty(n * 24, dtype=torch.uint8, device="cuda")
        sh = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
        rc = L.load().vx_render_primary_noalloc(C.byref(view), C.byref(cam), C.byref(p),
                                                C.c_void_p(rec.data_ptr()),
                                                C.c_void_p(sh.data_ptr()), C.c_void_p(0))
        assert rc == 0, L.load().vx_last_error()
        torch.cuda.synchronize()
        assert_records(vg.records(rec), fr["expect"], f"noalloc frame {fr['world']}")


@pytest.mark.gpu
def test_learned_frames_match_golden_except_steps(device_worlds):
    """The learned form (verification only: no network) on the golden
    cameras gives the golden records in every field but steps."""
    import torch
    import voxelg_b200 as vg
    from voxelg_b200 import learned as vl
    for fr in GOLDEN["frames"]:
        if fr["params"]["flags"] & 8:
            continue  # the learned form runs without the beam pre-pass
        dw = device_worlds[fr["world"]]
        cam, p = camera_of(fr["camera"], True), params_of(fr["params"], True)
        plain, _ = vg.render_primary(dw, cam, p)
        rec = torch.empty_like(plain)
        vl.render_learned(dw, None, cam, p, rec)
        torch.cuda.synchronize()
        assert_records(vg.records(rec), fr["expect"], f"learned frame {fr['world']}",
                       steps=False)


@pytest.mark.gpu
def test_pick_kernel_matches_golden(device_worlds):
    import voxelg_b200 as vg
    by_world = {}
    for pk in GOLDEN["picks"]:
        by_world.setdefault(pk["world"], []).append(pk)
    for name, pks in by_world.items():
        cams = np.array([pk["cam"] for pk in pks], np.float32)
        dirs = np.array([pk["dir"] for pk in pks], np.float32)
        out, hit = vg.raycast_batch(device_worlds[name], cams, dirs, origin=WORLDS[name]["origin"])
        for i, pk in enumerate(pks):
            e = pk["expect"]
            assert bool(hit[i]) == (e is not None), (pk, hit[i])
            if e is not None:
                assert list(out[i]["voxel"]) == e["voxel"], (pk, out[i])
                assert list(out[i]["normal"]) == e["normal"], (pk, out[i])
