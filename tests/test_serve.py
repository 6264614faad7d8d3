"""The ray-query serving loop, in both modes (continuous batching over
device slots; the device-resident request loop): results equal vx_trace
alone and the oracle, edits ordered in the request stream, the resident
loop's idle exit and restart, and the open-loop load generator."""
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


@pytest.mark.parametrize("resident,slots,budget", [
    (False, 4, 64 << 20), (False, 1, 8 << 20), (False, 8, 4 << 20),
    # the resident loop: ample budget, and one the 120 requests overrun (the
    # staging ring wraps and admission waits for completions)
    (True, 1, 64 << 20), (True, 1, 2 << 20)])
def test_batched_results_equal_alone(env, resident, slots, budget, c1_oracle_world):
    """Each request's records in the mix equal the same rays traced alone
    (vx_trace) and the oracle."""
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params(vg._lib.VX_F_L4 | vg._lib.VX_F_LUT | vg._lib.VX_F_LOD)
    srv = sv.Server(dw, p, mem_budget_bytes=budget, slots=slots, resident=resident)
    rng = np.random.default_rng(slots + 10 * resident + budget % 7)
    cap = min(20000, budget // slots // 56)
    reqs = [query_rays(rng, int(n)) for n in
            np.minimum(np.exp(rng.uniform(0, np.log(cap), 120)).astype(int) + 1, cap)]
    tickets = [srv.submit(r) for r in reqs]
    outs = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert st["requests"] == len(reqs) and st["rays"] == sum(len(r) for r in reqs)
    # slots: batches launched; resident: launches of the loop
    assert st["batches"] < len(reqs) or slots == 1, "requests were never batched together"
    if resident:
        assert 1 <= st["batches"] < len(reqs)
        assert st["peak_inflight_rays"] <= budget // 56
    for r, o in zip(reqs, outs):
        alone = vg.records(vg.trace(dw, r, p))
        assert np.array_equal(o.view(np.uint8), alone.view(np.uint8))
    for r, o in list(zip(reqs, outs))[:10]:
        want = po.trace_batch(c1_oracle_world, r, p)[0]
        assert np.array_equal(o.view(np.uint8), want.view(np.uint8))
    srv.close()


@pytest.mark.parametrize("resident", [False, True])
def test_edits_are_ordered_between_requests(env, resident):
    """A request submitted before an edit sees the old world, one submitted
    after it the new world, while both are in the same stream of work."""
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params(vg._lib.VX_F_L4)
    # a private world so the module world stays untouched
    w2 = vg.DeviceWorld(128, 64, 128)
    w2.upload(dw.download())
    srv = sv.Server(w2, p, slots=2, resident=resident)
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


@pytest.mark.parametrize("resident", [False, True])
def test_rejects_request_larger_than_slot(env, resident):
    import voxelg_b200.serve as sv
    vg, dw = env
    srv = sv.Server(dw, vg.default_params(), mem_budget_bytes=56 * 1000, slots=1,
                    resident=resident)
    with pytest.raises(vg._lib.VxError) as e:
        srv.submit(query_rays(np.random.default_rng(0), 1001))
    assert e.value.code == vg._lib.VX_ERR_BUSY
    # a request that fits still runs
    r = query_rays(np.random.default_rng(1), 1000)
    o = srv.wait(srv.submit(r))
    assert np.array_equal(o.view(np.uint8), vg.records(vg.trace(dw, r, vg.default_params())).view(np.uint8))
    srv.close()


@pytest.mark.parametrize("resident", [False, True])
def test_many_edits_interleaved_with_requests(env, resident):
    """Six rounds of mixed-size requests, each round followed by an edit of
    random bricks: every request's records equal the rays traced on a second
    world that received the same edits in the same order up to that request
    (for the resident loop: a fence, a drained launch and a restart per
    edit)."""
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params(vg._lib.VX_F_L4 | vg._lib.VX_F_LUT | vg._lib.VX_F_LOD)
    arrays = dw.download()
    w_srv = vg.DeviceWorld(128, 64, 128)
    w_ref = vg.DeviceWorld(128, 64, 128)
    w_srv.upload(arrays)
    w_ref.upload(arrays)
    srv = sv.Server(w_srv, p, mem_budget_bytes=32 << 20, resident=resident)
    rng = np.random.default_rng(21 + resident)
    n_bricks = 128 * 64 * 128
    live = []
    try:
        for rnd in range(6):
            for n in (1, 37, 512, 3000, 64):
                r = query_rays(rng, n)
                live.append((srv.submit(r), vg.records(vg.trace(w_ref, r, p)).copy()))
            k = 2000
            idx = rng.choice(n_bricks, k, replace=False).astype(np.uint32)
            bricks = np.zeros(k, po.BRICK)
            occ = rng.integers(0, 2**63, k, dtype=np.uint64) | rng.integers(0, 2, k, dtype=np.uint64)
            bricks["occupancy"] = occ
            bits = ((occ[:, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(bool)
            bricks["materials"] = np.where(bits, rng.choice(np.array([2, 3, 4, 12], np.uint8), (k, 64)), 0)
            srv.edit(idx, bricks)
            w_ref.apply_dirty(idx, bricks)
        for t, want in live:
            got = srv.wait(t)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
        assert srv.stats()["edits"] == 6
    finally:
        srv.close()
        w_srv.close()
        w_ref.close()


def pinned(n, dtype):
    """A numpy array of n elements in page-locked host memory."""
    import torch
    buf = torch.empty(n * dtype.itemsize, dtype=torch.uint8, pin_memory=True)
    return buf, buf.numpy().view(dtype)


def test_resident_reads_and_writes_page_locked_buffers_in_place(env, c1_oracle_world):
    """Page-locked request buffers are read and written by the loop itself
    (no staging): records equal vx_trace alone and the oracle."""
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params(vg._lib.VX_F_L4 | vg._lib.VX_F_LUT | vg._lib.VX_F_LOD)
    srv = sv.Server(dw, p, mem_budget_bytes=32 << 20, resident=True)
    rng = np.random.default_rng(5)
    keep, live = [], []
    for n in (1, 31, 32, 33, 4096, 20000):
        hold_r, rays = pinned(n, vg._lib.RAY_DTYPE)
        rays[:] = query_rays(rng, n).view(vg._lib.RAY_DTYPE)
        hold_o, out = pinned(n, vg._lib.RECORD_DTYPE)
        out.view(np.uint8)[:] = 0xAB
        keep += [hold_r, hold_o]
        live.append((rays, out, srv.submit(rays, out)))
    for rays, out, t in live:
        got = srv.wait(t)
        assert got is out
        alone = vg.records(vg.trace(dw, rays, p))
        assert np.array_equal(out.view(np.uint8), alone.view(np.uint8))
    rays, out, _ = live[3]
    want = po.trace_batch(c1_oracle_world, np.asarray(rays).view(po.RAY), p)[0]
    assert np.array_equal(out.view(np.uint8), want.view(np.uint8))
    # page-locked but not 16-byte aligned: records 24 bytes into their buffer
    # go through staging while the (aligned) rays are read in place
    hold_r, rays = pinned(1000, vg._lib.RAY_DTYPE)
    rays[:] = query_rays(rng, 1000).view(vg._lib.RAY_DTYPE)
    hold_o, out_all = pinned(1001, vg._lib.RECORD_DTYPE)
    out = out_all[1:]
    assert out.ctypes.data % 16 == 8
    got = srv.wait(srv.submit(rays, out))
    assert got is out
    alone = vg.records(vg.trace(dw, rays, p))
    assert np.array_equal(out.view(np.uint8), alone.view(np.uint8))
    srv.close()


def test_resident_loop_ends_when_idle_and_restarts(env):
    """The loop's idle wait runs out (idle_us = 100): the launch ends, and the
    next request starts another one; results are unaffected."""
    import time
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params()
    srv = sv.Server(dw, p, mem_budget_bytes=16 << 20, resident=True, idle_us=100)
    rng = np.random.default_rng(9)
    for k in range(4):
        r = query_rays(rng, 500 + k)
        o = srv.wait(srv.submit(r))
        assert np.array_equal(o.view(np.uint8), vg.records(vg.trace(dw, r, p)).view(np.uint8))
        time.sleep(0.02)  # 200x the idle time
    st = srv.stats()
    assert st["requests"] == 4 and st["batches"] == 4, st
    srv.close()


def test_resident_wait_limit_stops_the_server_and_leaves_the_device_usable(env):
    """A warp's wait for work is bounded.  With wait_us (1 ms) far below
    idle_us (200 ms), the idle workers' waits run out while the launch is
    still up: each records the loop's error word and returns, the server
    stops with VX_ERR_DEVICE, and the device keeps working."""
    import time
    import voxelg_b200.serve as sv
    vg, dw = env
    p = vg.default_params()
    srv = sv.Server(dw, p, mem_budget_bytes=16 << 20, resident=True, idle_us=200000,
                    wait_us=1000)
    r = query_rays(np.random.default_rng(11), 64)
    o = srv.wait(srv.submit(r))  # served well inside the limit
    alone = vg.records(vg.trace(dw, r, p))
    assert np.array_equal(o.view(np.uint8), alone.view(np.uint8))
    time.sleep(0.1)
    with pytest.raises(vg._lib.VxError) as e:
        srv.submit(r)
    assert e.value.code == vg._lib.VX_ERR_DEVICE
    assert "wait" in str(e.value)
    srv.close()
    # the context is intact
    again = vg.records(vg.trace(dw, r, p))
    assert np.array_equal(again.view(np.uint8), alone.view(np.uint8))


@pytest.mark.parametrize("resident", [False, True])
def test_load_generator_short_run(env, resident):
    import voxelg_b200.serve as sv
    vg, dw = env
    w2 = vg.DeviceWorld(128, 64, 128)
    w2.upload(dw.download())
    srv = sv.Server(w2, vg.default_params(), mem_budget_bytes=256 << 20, slots=4,
                    resident=resident)
    st = srv.bench(clients=16, rate_per_client=100.0, seconds=1.0, max_rays=20000,
                   edit_fraction_per_s=0.01)
    assert st["requests"] > 500 and st["rays"] > 0 and st["edits"] > 10
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    srv.close()
    w2.close()
