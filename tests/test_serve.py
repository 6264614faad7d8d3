"""The ray-query serving loop: continuous batching over device slots, edits
ordered in the request stream, and the open-loop load generator."""
import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200 as vg
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    yield vg, dw
    dw.close()


def query_rays(rng, n, vox=(512, 256, 512)):
    r = np.zeros(n, po.RAY)
    r["org"] = rng.uniform([0, 0, 0], vox, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    r["dir"] = d
    r["tmax"] = rng.choice(np.array([8.0, 32.0, 128.0, 512.0], np.float32), n)
    r["kind"] = rng.choice(np.array([0, 0, 0, 1], np.uint32), n)
    return r


@pytest.mark.parametrize("slots,budget", [(4, 64 << 20), (1, 8 << 20), (8, 4 << 20)])
def test_batched_results_equal_alone(env, slots, budget, c1_oracle_world):
    """Each request's records in the mix equal the same rays traced alone
    (vx_trace) and the oracle."""
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params(vg._lib.VX_F_L4 | vg._lib.VX_F_LUT | vg._lib.VX_F_LOD)
    srv = sv.Server(dw, p, mem_budget_bytes=budget, slots=slots)
    rng = np.random.default_rng(slots)
    cap = min(20000, budget // slots // 56)
    reqs = [query_rays(rng, int(n)) for n in
            np.minimum(np.exp(rng.uniform(0, np.log(cap), 120)).astype(int) + 1, cap)]
    tickets = [srv.submit(r) for r in reqs]
    outs = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert st["requests"] == len(reqs) and st["rays"] == sum(len(r) for r in reqs)
    assert st["batches"] < len(reqs) or slots == 1, "requests were never batched together"
    for r, o in zip(reqs, outs):
        alone = vg.records(vg.trace(dw, r, p))
        assert np.array_equal(o.view(np.uint8), alone.view(np.uint8))
    for r, o in list(zip(reqs, outs))[:10]:
        want = po.trace_batch(c1_oracle_world, r, p)[0]
        assert np.array_equal(o.view(np.uint8), want.view(np.uint8))
    srv.close()


def test_edits_are_ordered_between_requests(env):
    """A request submitted before an edit sees the old world, one submitted
    after it the new world, while both are in the same stream of work."""
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params(vg._lib.VX_F_L4)
    # a private world so the module world stays untouched
    w2 = vg.DeviceWorld(128, 64, 128)
    w2.upload(dw.download())
    srv = sv.Server(w2, p, slots=2)
    n = 4096
    rays = np.zeros(n, po.RAY)
    rays["org"] = np.array([256.0, 250.0, 256.0], np.float32)
    rays["dir"] = np.array([0.0, -1.0, 0.0], np.float32)
    rays["org"][:, 0] += np.arange(n) % 64
    rays["org"][:, 2] += np.arange(n) // 64
    rays["tmax"] = 700.0
    before = vg.records(vg.trace(w2, rays, p)).copy()
    # a stone slab at y = 200 over the queried columns
    bricks = np.zeros(16 * 16, po.BRICK)
    bricks["occupancy"] = np.uint64(0xFFFFFFFFFFFFFFFF)
    bricks["materials"] = 4
    idx = np.array([(256 // 4 + i) + (200 // 4) * 128 + (256 // 4 + k) * 128 * 64
                    for k in range(16) for i in range(16)], np.uint32)
    t1 = srv.submit(rays)
    srv.edit(idx, bricks)
    t2 = srv.submit(rays)
    o1, o2 = srv.wait(t1), srv.wait(t2)
    assert np.array_equal(o1.view(np.uint8), before.view(np.uint8))
    assert (o2["voxel"][:, 1] == 203).all() and (o2["mat"] == 4).all()
    after = vg.records(vg.trace(w2, rays, p))
    assert np.array_equal(o2.view(np.uint8), after.view(np.uint8))
    assert srv.stats()["edits"] == 1
    srv.close()
    w2.close()


def test_rejects_request_larger_than_slot(env):
    import voxelg_b200.serve as sv
    vg, dw = env
    srv = sv.Server(dw, vg.default_params(), mem_budget_bytes=56 * 1000, slots=1)
    with pytest.raises(vg._lib.VxError) as e:
        srv.submit(query_rays(np.random.default_rng(0), 1001))
    assert e.value.code == vg._lib.VX_ERR_BUSY
    srv.close()


def test_load_generator_short_run(env):
    import voxelg_b200.serve as sv
    vg, dw = env
    w2 = vg.DeviceWorld(128, 64, 128)
    w2.upload(dw.download())
    srv = sv.Server(w2, vg.default_params(), mem_budget_bytes=256 << 20, slots=4)
    st = srv.bench(clients=16, rate_per_client=100.0, seconds=1.0, max_rays=20000,
                   edit_fraction_per_s=0.01)
    assert st["requests"] > 500 and st["rays"] > 0 and st["edits"] > 10
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    srv.close()
    w2.close()
