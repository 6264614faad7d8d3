"""The learned start-distance proposal: the network oracle (CPU), the device
features / FP32 gradients / BF16 inference against it, on-device training,
and the learned frame -- records equal to the plain DDA's on every ray, with
fewer DDA iterations."""
import math

import numpy as np
import pytest

from oracle import mlp as om
from oracle import pyoracle as po

F_METHOD = 1 | 2 | 4  # L4 | LUT | LOD


# ------------------------------------------------------------------ CPU
def test_oracle_gradient_matches_finite_differences():
    """Pins the oracle's backward pass: central differences in float64."""
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, om.N_PARAMS)
    X = rng.uniform(-1, 1, (16, om.N_IN))
    X[:, 70:] = 0.0
    y = rng.uniform(2, 6, 16)
    loss, g = om.loss_and_grad(p, X, y)
    idx = rng.choice(om.N_PARAMS, 64, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        num = (om.loss_and_grad(p + e, X, y)[0] - om.loss_and_grad(p - e, X, y)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_oracle_features_layout():
    org = np.array([[0.5, 70.25, 130.0], [-1.0, 10.0, 511.75]], np.float32)
    d = np.array([[0.0, -1.0, 0.0], [0.6, 0.0, 0.8]], np.float32)
    w = np.array([0x8000000000000001, 0x2], np.uint64)
    f = om.features(org, d, w)
    assert f.shape == (2, 80) and np.all(f[:, 70:] == 0)
    assert np.allclose(f[0, :3], [0.5 / 64, 6.25 / 64, 2.0 / 64])
    assert np.allclose(f[1, :3], [63.0 / 64, 10.0 / 64, 63.75 / 64])
    assert f[0, 6] == 1 and f[0, 69] == 1 and f[0, 7:69].sum() == 0
    assert f[1, 7] == 1 and f[1, 6:70].sum() == 1


def test_default_config_and_null_arguments():
    from voxelg_b200 import _lib as L
    from voxelg_b200 import learned as vl
    c = vl.default_config()
    assert (c.poses, c.rays_per_pose, c.steps, c.batch) == (200, 81920, 3000, 16384)
    assert c.poses * c.rays_per_pose >= 16_000_000
    assert c.flags == F_METHOD and (c.width, c.height) == (1920, 1080)
    lib = L.load()
    assert lib.vx_proposal_create(None, 1, None) == L.VX_ERR_INVALID
    assert lib.vx_proposal_destroy(None) == L.VX_OK
    assert lib.vx_proposal_get_params(None, None, 0) == L.VX_ERR_INVALID
    assert lib.vx_render_learned(None, None, None, None, 1.0, None, None, None) == \
        L.VX_ERR_INVALID


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200 as vg
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    yield vg, dw, cfg
    dw.close()


@pytest.fixture(scope="module")
def trained(env):
    """A proposal trained with a reduced schedule (the full one runs in the
    benchmark)."""
    from voxelg_b200 import learned as vl
    vg, dw, _ = env
    prop = vl.Proposal(dw, seed=7)
    c = vl.default_config(poses=60, rays_per_pose=32768, steps=1200, seed=5)
    curve, before, after = prop.train(dw, c)
    yield prop, curve, before, after
    prop.close()


def _rays(rng, n, vox=(512, 256, 512)):
    r = np.zeros(n, po.RAY)
    r["org"] = rng.uniform([0, 60, 0], [vox[0], 220, vox[2]], size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    r["dir"] = d
    r["tmax"] = 700.0
    return r


@pytest.mark.gpu
def test_device_features_equal_oracle(env, c1_oracle_world):
    from voxelg_b200 import learned as vl
    vg, dw, cfg = env
    prop = vl.Proposal(dw, seed=1)
    rng = np.random.default_rng(1)
    rays = _rays(rng, 5000)
    rays["org"][:10] = [[-5.0, 10.0, 10.0]] * 10      # outside the window: zero bits
    f = prop.features(dw, rays).cpu().numpy()
    words = om.origin_chunk_words(c1_oracle_world.a["chunk_mask"], cfg.bricks, rays["org"])
    want = om.features(rays["org"], rays["dir"], words)
    assert np.array_equal(f, want)
    assert np.all(f[:10, 6:70] == 0) and f[10:, 6:70].sum() > 0
    prop.close()


@pytest.mark.gpu
def test_gradients_match_oracle(env):
    """FP32 device forward/backward against the float64 oracle.  Tolerance:
    loss relative 1e-5; per parameter tensor, max |g_dev - g_ref| <= 1e-3 *
    max |g_ref| + 1e-7 (fp32 sums in a different order, atomics)."""
    import torch
    from voxelg_b200 import learned as vl
    vg, dw, _ = env
    prop = vl.Proposal(dw, seed=3)
    p = prop.params().astype(np.float64)
    assert np.all(om.unpack(p)["W1"][:, 70:] == 0)
    rng = np.random.default_rng(3)
    for B in (1, 37, 4096):
        X = rng.uniform(-1, 1, (B, om.N_IN)).astype(np.float32)
        X[:, 70:] = 0
        X[:, 6:70] = rng.integers(0, 2, (B, 64))
        y = rng.uniform(1, 6.5, B).astype(np.float32)
        loss, g = prop.grad(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda())
        rl, rg = om.loss_and_grad(p.astype(np.float32).astype(np.float64), X, y)
        assert abs(loss - rl) <= 1e-5 * abs(rl) + 1e-7, (B, loss, rl)
        o = 0
        for name, shape in om.SIZES:
            n = int(np.prod(shape))
            a, b = g[o:o + n], rg[o:o + n]
            assert np.max(np.abs(a - b)) <= 1e-3 * np.max(np.abs(b)) + 1e-7, (B, name)
            o += n
    prop.close()


@pytest.mark.gpu
def test_bf16_inference_matches_oracle(env, trained):
    """BF16 tensor-core inference against the float64 forward with the same
    parameters.  Tolerance: |y_dev - y_ref| <= 0.1 + 0.02 |y_ref| in log t
    (at most ~12% in distance): the operands of all three 64-wide layers are
    rounded to bf16 (8 significant bits) and tanh is the hardware
    approximation; the value only bounds the verification walk."""
    vg, dw, _ = env
    prop = trained[0]
    rng = np.random.default_rng(4)
    rays = _rays(rng, 20000 + 7)       # not a multiple of the 16-ray pass
    f = prop.features(dw, rays)
    y = prop.infer(f).cpu().numpy()
    ref, _ = om.forward(prop.params().astype(np.float64), f.cpu().numpy())
    err = np.abs(y - ref)
    assert np.all(err <= 0.1 + 0.02 * np.abs(ref)), float(err.max())


@pytest.mark.gpu
def test_training_reduces_held_out_loss(trained):
    _, curve, before, after = trained
    assert np.all(np.isfinite(curve))
    assert after < 0.5 * before, (before, after)
    assert curve[-100:].mean() < 0.5 * curve[:20].mean()


def _plain_and_learned(vg, dw, cam, flags, proposal, scale=1.0):
    import torch
    from voxelg_b200 import learned as vl
    p = vg.default_params(flags)
    plain, _ = vg.render_primary(dw, cam, p)
    rec = torch.empty_like(plain)
    st = vl.render_learned(dw, proposal, cam, p, rec, scale=scale)
    return vg.records(plain), vg.records(rec), st


def _same_but_steps(a, b):
    fa, fb = a.copy(), b.copy()
    fa["steps"] = 0
    fb["steps"] = 0
    return np.array_equal(fa.view(np.uint8), fb.view(np.uint8))


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["trained", "untrained", "none"])
def test_learned_frame_equals_plain_1080p(env, trained, which):
    """Every ray of the 1920x1080 frame of the 512x256x512 world: the learned
    form's records equal the plain DDA's except steps."""
    from voxelg_b200 import learned as vl
    vg, dw, _ = env
    prop = {"trained": trained[0], "untrained": None, "none": None}[which]
    if which == "untrained":
        prop = vl.Proposal(dw, seed=11)
    cam = vg.default_camera(dw, 1920, 1080)
    a, b, st = _plain_and_learned(vg, dw, cam, F_METHOD, prop)
    assert st.rays == 1920 * 1080 and st.fallback == 0
    assert _same_but_steps(a, b)
    assert st.iters == int(b["steps"].astype(np.int64).sum())
    if which == "untrained":
        prop.close()


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [0, 1, 2, 4, 1 | 2, 2 | 4, F_METHOD])
@pytest.mark.parametrize("pose", [((256, 140, 256), 0.0, -15.0), ((100.5, 97.3, 410.2), 2.1, -35.0),
                                  ((300.0, 60.0, 90.0), 4.0, 20.0), ((256, 250, 256), 0.3, -89.0),
                                  ((0.0, 130.0, 0.0), 0.785, -10.0)])
def test_learned_equals_plain_flags_and_poses(env, trained, flags, pose):
    vg, dw, _ = env
    pos, yaw, pitch = pose
    cam = vg.camera_from_pose(pos, yaw, math.radians(pitch), math.radians(70.0), 480, 270)
    for prop, scale in ((trained[0], 1.0), (trained[0], 0.5), (None, 1.0)):
        a, b, st = _plain_and_learned(vg, dw, cam, flags, prop, scale)
        assert _same_but_steps(a, b), (flags, pose, scale)


@pytest.mark.gpu
def test_learned_unaligned_window_and_oracle(env, trained, c1_oracle_world):
    """A window corner off the chunk grid runs the plain DDA inside the same
    kernel; the learned records also equal the oracle's except steps."""
    vg, dw, _ = env
    cam = vg.camera_from_pose((200.0, 150.0, 300.0), 1.0, math.radians(-20.0),
                              math.radians(70.0), 320, 180, world_origin=(5, 0, -3))
    a, b, st = _plain_and_learned(vg, dw, cam, F_METHOD, trained[0])
    assert _same_but_steps(a, b) and st.none == st.rays
    cam = vg.default_camera(dw, 320, 180)
    a, b, st = _plain_and_learned(vg, dw, cam, F_METHOD, trained[0])
    want = po.render_frame(c1_oracle_world, cam, po.default_params(F_METHOD))[0]
    assert _same_but_steps(b, want)
    assert np.array_equal(a.view(np.uint8), want.view(np.uint8))


def _batch_ms(frame, reps=20):
    """Mean ms per frame of `reps` frames enqueued back to back on the
    current stream between two CUDA events."""
    import torch
    st = torch.cuda.current_stream()
    for _ in range(3):
        frame()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        frame()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


@pytest.mark.gpu
def test_learned_gain_over_plain(env, trained):
    """What the learned form buys on the 1920x1080 frame: fewer DDA
    iterations per ray than the plain DDA with identical records, and more
    rays per second (frames enqueued back to back, the same way for both
    forms)."""
    import torch
    from voxelg_b200 import learned as vl
    vg, dw, _ = env
    cam = vg.default_camera(dw, 1920, 1080)
    p = vg.default_params(F_METHOD)
    a, b, st = _plain_and_learned(vg, dw, cam, F_METHOD, trained[0])
    plain_iters = int(a["steps"].astype(np.int64).sum())
    assert _same_but_steps(a, b)
    assert st.iters < 0.7 * plain_iters, (st.iters, plain_iters)
    assert st.miss > 0.2 * st.rays and st.none < 0.01 * st.rays
    rec = torch.empty(1920 * 1080 * 24, dtype=torch.uint8, device="cuda")
    plain_ms = min(_batch_ms(lambda: vg.render_primary(dw, cam, p, rec)) for _ in range(3))
    learned_ms = min(_batch_ms(lambda: vl.render_learned(dw, trained[0], cam, p, rec,
                                                         stats=False)) for _ in range(3))
    print(f"\nplain {plain_iters / st.rays:.2f} it/ray {plain_ms:.4f} ms; learned "
          f"{st.iters / st.rays:.2f} it/ray {learned_ms:.4f} ms ({plain_ms / learned_ms:.3f}x; "
          f"accepted {st.accepted / st.rays:.1%}, partial {st.partial / st.rays:.1%}, "
          f"miss {st.miss / st.rays:.1%})")
    assert learned_ms < 0.95 * plain_ms, (plain_ms, learned_ms)


@pytest.mark.gpu
def test_trained_network_predicts_first_hits(env, trained):
    """The network the learned form runs: on the benchmark frame, its
    per-block estimate of log first-hit distance (a miss counts as log tmax,
    the label it is trained on) has under 0.6x the mean squared error of an
    untrained network's.  The fixture's short training (1200 steps) still
    over-estimates near hits, so the error is measured over every block
    centre, hits and misses, as the training loss is.  The records stay the
    plain DDA's whatever the network predicts."""
    import torch
    from voxelg_b200 import learned as vl
    vg, dw, _ = env
    cam = vg.default_camera(dw, 1920, 1080)
    p = vg.default_params(F_METHOD)
    plain, _ = vg.render_primary(dw, cam, p)
    torch.cuda.synchronize()
    a = vg.records(plain)
    W, H, tmax = 1920, 1080, 700.0
    # block centre rays of the 16x8 proposal blocks, as features
    bx, by = np.meshgrid(np.arange(W // 16), np.arange(H // 8))
    px = (bx * 16 + 8).ravel()
    py = (by * 8 + 4).ravel()
    r = a.reshape(H, W)[py, px]
    hit = (r["flags"] & 1) != 0
    target = np.where(hit, np.log(np.maximum(r["t"], 1e-3)), np.log(tmax))
    rays = np.zeros(len(px), po.RAY)
    rays["org"] = np.array(list(cam.origin), np.float32)
    rays["dir"] = np.stack([np.array(po.ray_dir_uv(cam, (x + 0.5) / W, (y + 0.5) / H),
                                     np.float32) for x, y in zip(px, py)])
    rays["tmax"] = tmax
    untrained = vl.Proposal(dw, seed=11)
    mse = {}
    for name, prop in (("trained", trained[0]), ("untrained", untrained)):
        y = prop.infer(prop.features(dw, rays)).cpu().numpy()
        mse[name] = float(np.mean((y - target) ** 2))
    untrained.close()
    print(f"\nmean squared log t error over {len(px)} block centres "
          f"({hit.mean():.0%} hits): {mse}")
    assert mse["trained"] < 0.6 * mse["untrained"], mse


@pytest.mark.gpu
def test_learned_equals_plain_on_the_2048_world(env, trained):
    """The 2048x256x2048 benchmark world, where rays reach the tile LOD
    distance (520) inside the window: the learned form (proofs capped before
    tile_lod_t in brick cubes) gives the plain DDA's records except steps,
    for several poses and flag sets."""
    vg, dw_c1, _ = env
    cfg = vg.CONFIGS["c2"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    try:
        for pos, yaw, pitch in (((1024.0, 140.0, 1024.0), 0.0, -15.0),
                                ((300.5, 180.25, 1900.75), 2.4, -6.0),
                                ((1700.0, 230.0, 200.0), 4.1, -3.0)):
            cam = vg.camera_from_pose(pos, yaw, math.radians(pitch), math.radians(70.0), 640, 360)
            for flags in (F_METHOD, 1 | 4, 4):
                a, b, st = _plain_and_learned(vg, dw, cam, flags, None)
                assert _same_but_steps(a, b), (pos, flags)
                assert st.none < 0.01 * st.rays
    finally:
        dw.close()


@pytest.mark.gpu
def test_learned_iteration_cap_falls_back(env, trained):
    """With a small iteration cap the restarted walks' inflated counters
    reach it and the plain DDA decides those rays: records still equal."""
    vg, dw, _ = env
    cam = vg.default_camera(dw, 480, 270)
    for cap in (6, 12, 20):
        p = vg.default_params(F_METHOD)
        p.max_iters = cap
        import torch
        from voxelg_b200 import learned as vl
        plain, _ = vg.render_primary(dw, cam, p)
        rec = torch.empty_like(plain)
        st = vl.render_learned(dw, trained[0], cam, p, rec)
        assert _same_but_steps(vg.records(plain), vg.records(rec)), cap
        assert st.fallback > 0, cap
