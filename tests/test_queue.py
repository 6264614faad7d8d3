"""The mixed ray queue: primary rays that spawn their shadow ray, GI-probe
rays, picking rays, shuffled, traced by one persistent launch (also
captured in a CUDA graph) -- bit-exact against the oracle for every tuning
the autotuner tries."""
import numpy as np
import pytest

from oracle import pyoracle as po

DIMS = (128, 64, 128)


def small_queue(vg, seed=2, w=160, h=90):
    import voxelg_b200.queue as q
    cam = vg.default_camera(DIMS, w, h)
    rays, counts = q.mixed_queue(DIMS, cam, w, h, seed, probe_radius=48, pick_rays=3000)
    return cam, rays, counts


def test_workload_generator():
    import voxelg_b200 as vg
    import voxelg_b200.queue as q
    cam = vg.default_camera(DIMS, 1920, 1080)
    rays, c = q.mixed_queue(DIMS, cam, 1920, 1080, 1)
    assert c["primary"] == 2073600 and c["probes"] == 32 * 16 * 32 and c["picking"] == 10000
    assert len(rays) == c["primary"] + c["gi_probe"] + c["picking"]
    d = rays["dir"].astype(np.float64)
    assert np.abs(np.linalg.norm(d, axis=1) - 1).max() < 1e-6
    assert set(np.unique(rays["tmax"])) == {8.0, 256.0, 700.0}
    assert (rays["kind"][rays["tmax"] == 700.0] == vg._lib.VX_RAY_SPAWN_SHADOW).all()
    fd = q.fibonacci_dirs(64)
    assert len(np.unique(np.round(fd, 5), axis=0)) == 64
    # shuffled: primaries are spread over the queue
    first = np.flatnonzero(rays["tmax"] == 700.0)
    assert first.min() < 100 and first.max() > len(rays) - 100


def test_oracle_queue_primary_equals_frame(c1_oracle_world):
    """A queue primary ray is the frame's pixel ray without the beam skip:
    the oracle gives it the same record."""
    import voxelg_b200 as vg
    import voxelg_b200.queue as q
    cam = vg.default_camera(DIMS, 64, 36)
    p = po.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD)
    rays = np.zeros(64 * 36, po.RAY)
    rays["org"] = np.array(list(cam.origin), np.float32)
    rays["dir"] = q.primary_dirs(cam, 64, 36)
    rays["tmax"] = 700.0
    rays["kind"] = 256
    rec, sh, _, _ = po.trace_batch(c1_oracle_world, rays, p, shadows=True)
    frame = po.render_frame(c1_oracle_world, cam, p)[0]
    assert np.array_equal(rec.view(np.uint8), frame.view(np.uint8))
    hit = (rec["flags"] & 1) == 1
    assert np.array_equal(sh["traced"] == 1, hit) and hit.any()


@pytest.fixture(scope="module")
def gpu(c1_oracle_world):
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
def test_queue_bit_exact_every_tuning(gpu, c1_oracle_world):
    import torch
    import voxelg_b200.queue as q
    vg, dw = gpu
    cam, rays, counts = small_queue(vg)
    for flags in (po.OR_F_L4, po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD):
        p = vg.default_params(flags, frame=3.0)
        want, wsh, _, _ = po.trace_batch(c1_oracle_world, rays, p, shadows=True)
        assert (wsh["traced"] == 1).sum() > 1000
        for bt, rm, so in ((128, 32, 1), (64, 1, 0), (256, 16, 1), (128, 8, 0)):
            t = q.default_tuning()
            t.block_threads, t.refill_min, t.sort = bt, rm, so
            _, out, sh = q.run(dw, rays, p, tuning=t)
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy(), want.view(np.uint8)), (flags, bt, rm, so)
            assert np.array_equal(sh.cpu().numpy(), wsh.view(np.uint8)), (flags, bt, rm, so)


@pytest.mark.gpu
def test_queue_autotune_and_graph(gpu, c1_oracle_world):
    import torch
    import voxelg_b200.queue as q
    vg, dw = gpu
    cam, rays, counts = small_queue(vg, seed=5)
    p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD)
    best, ms, rt, out, sh = q.autotune(dw, rays, p, reps=2)
    assert ms > 0 and best.block_threads in (64, 128, 256) and 1 <= best.refill_min <= 32
    want, wsh, _, _ = po.trace_batch(c1_oracle_world, rays, p, shadows=True)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want.view(np.uint8))
    g = q.Graph(dw, rt, p, tuning=best)
    for _ in range(3):
        g.out.zero_()
        g.launch()
        torch.cuda.synchronize()
        assert np.array_equal(g.out.cpu().numpy(), want.view(np.uint8))
        assert np.array_equal(g.shadow.cpu().numpy(), wsh.view(np.uint8))
    g.close()


@pytest.mark.gpu
def test_queue_edge_rays(gpu, c1_oracle_world):
    """Rays outside the window, zero-length budgets, axis-aligned and every
    kind with and without the spawn flag."""
    import torch
    import voxelg_b200.queue as q
    vg, dw = gpu
    rng = np.random.default_rng(8)
    n = 20000
    rays = np.zeros(n, po.RAY)
    rays["org"] = rng.uniform([-60, -30, -60], [572, 300, 572], size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[::7, 0] = 0.0
    d[::11] = np.array([0.0, -1.0, 0.0], np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    rays["dir"] = d
    rays["tmax"] = rng.choice(np.array([0.0, 8.0, 256.0, 700.0], np.float32), n)
    rays["kind"] = rng.choice(np.array([0, 1, 2, 256, 257, 258, 3], np.uint32), n)
    p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD)
    want, wsh, _, _ = po.trace_batch(c1_oracle_world, rays, p, shadows=True)
    for so in (0, 1):
        t = q.default_tuning()
        t.block_threads, t.refill_min, t.sort = 256, 32, so
        _, out, sh = q.run(dw, rays, p, tuning=t)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want.view(np.uint8)), so
        assert np.array_equal(sh.cpu().numpy(), wsh.view(np.uint8)), so


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 31, 33, 2047, 2048, 2049, 6149])
def test_queue_sorted_sizes(gpu, c1_oracle_world, n):
    """The radix-sorted queue at sizes around its 2048-ray tiles and the
    32-lane packets: every record equals the oracle's."""
    import torch
    import voxelg_b200.queue as q
    vg, dw = gpu
    rng = np.random.default_rng(n)
    rays = np.zeros(n, po.RAY)
    rays["org"] = rng.uniform([0, 60, 0], [512, 220, 512], size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    rays["dir"] = d
    rays["tmax"] = 300.0
    rays["kind"] = rng.choice(np.array([0, 1, 2, 256], np.uint32), n)
    p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD)
    want, wsh, _, _ = po.trace_batch(c1_oracle_world, rays, p, shadows=True)
    t = q.default_tuning()
    t.block_threads, t.refill_min, t.sort = 128, 32, 1
    _, out, sh = q.run(dw, rays, p, tuning=t)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want.view(np.uint8))
    assert np.array_equal(sh.cpu().numpy(), wsh.view(np.uint8))
