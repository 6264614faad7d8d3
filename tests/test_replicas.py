"""World replicas across ranks: the dirty set of an edit made on one rank
reaches every rank unchanged and leaves every replica identical
(voxelg_b200.replicas; the upload set of renderer.rs:1345-1394)."""
import hashlib
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from oracle import pyoracle as po

DIMS = (64, 16, 64)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dirty_set(seed, n=300):
    """Random bricks (materials where the occupancy bit is set) at indices
    with repeats, so that the last occurrence must win."""
    rng = np.random.default_rng(seed)
    nb = DIMS[0] * DIMS[1] * DIMS[2]
    idx = rng.integers(0, nb, n).astype(np.uint32)
    k = min(20, n // 4)
    idx[n // 2:n // 2 + k] = idx[:k]
    b = np.zeros(n, po.BRICK)
    occ = rng.integers(0, 2, (n, 64)).astype(np.uint64)
    occ[::7] = 1                                     # some full, uniform bricks
    b["occupancy"] = np.bitwise_or.reduce(occ << np.arange(64, dtype=np.uint64), axis=1)
    mats = rng.choice(np.array([2, 3, 4, 14, 18, 33], np.uint8), (n, 64))
    mats[::7] = 4
    b["materials"] = np.where(occ == 1, mats, 0).astype(np.uint8)
    return idx, b


def _apply_to(w: po.World):
    def apply(idx, bricks):
        for i, b in zip(idx, bricks):                # in order: the last one wins
            w.a["bricks"][i] = b
        w.rebuild()
    return apply


def _digest(w: po.World) -> str:
    h = hashlib.sha256()
    for k in po.World.NAMES:
        h.update(np.ascontiguousarray(w.a[k]).view(np.uint8).tobytes())
    return h.hexdigest()


def _rank(rank, world_size, port, q, n):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world_size))
    import torch.distributed as dist

    from voxelg_b200.replicas import broadcast_dirty
    dist.init_process_group("gloo", rank=rank, world_size=world_size,
                            timeout=timedelta(seconds=60))
    try:
        w = po.World(*DIMS)
        idx, b = _dirty_set(5, n) if rank == 1 else (None, None)
        got_idx, got_b = broadcast_dirty(None, idx, b, src=1, apply=_apply_to(w))
        # a second edit from the other rank, in the same order on both
        idx2, b2 = _dirty_set(6, 40) if rank == 0 else (None, None)
        broadcast_dirty(None, idx2, b2, src=0, apply=_apply_to(w))
        q.put((rank, hashlib.sha256(got_idx.tobytes() + got_b.tobytes()).hexdigest(),
               _digest(w)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [300, 0])
def test_two_ranks_end_with_identical_replicas(n):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q, n)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    # what one process gets by applying both edits itself
    w = po.World(*DIMS)
    idx, b = _dirty_set(5, n) if n else (np.zeros(0, np.uint32), np.zeros(0, po.BRICK))
    if n:
        _apply_to(w)(idx, b)
    _apply_to(w)(*_dirty_set(6, 40))
    sent = hashlib.sha256(idx.tobytes() + b.tobytes()).hexdigest()
    assert got[0][1:] == got[1][1:] == (sent, _digest(w))


def test_src_length_mismatch_raises_before_any_collective():
    import torch.distributed as dist

    from voxelg_b200.replicas import broadcast_dirty
    port = _free_port()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1, timeout=timedelta(seconds=30))
    try:
        idx, b = _dirty_set(1, 10)
        with pytest.raises(ValueError):
            broadcast_dirty(None, idx, b[:9], src=0)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_nccl_replica_matches_oracle():
    """One NCCL rank: the set goes through device buffers and
    vx_world_apply_dirty, and the device world equals the oracle's with the
    same bricks applied in order."""
    import torch
    import torch.distributed as dist

    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200 as vg
    from voxelg_b200.replicas import broadcast_dirty
    torch.cuda.set_device(0)
    port = _free_port()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1, timeout=timedelta(seconds=60))
    try:
        dw = vg.DeviceWorld(*DIMS)
        ow = po.World(*DIMS)
        for seed in (5, 6):
            idx, b = _dirty_set(seed)
            broadcast_dirty(dw, idx, b, src=0)
            _apply_to(ow)(idx, b)
        torch.cuda.synchronize()
        got = dw.download()
        for k in po.World.NAMES:
            assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8),
                                  np.ascontiguousarray(ow.a[k]).view(np.uint8)), k
        cam = vg.camera_from_pose((128.0, 50.0, 20.0), 0.3, -0.4, 1.2, 96, 54)
        p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM)
        rec, _ = vg.render_primary(dw, cam, p)
        torch.cuda.synchronize()
        want = po.render_frame(ow, cam, p)[0]
        assert np.array_equal(vg.records(rec).view(np.uint8), want.view(np.uint8))
        dw.close()
    finally:
        dist.destroy_process_group()


# ------------------------------------------------------ one frame split by rows
def test_split_rows_cover_every_row_once():
    from voxelg_b200.replicas import split_rows
    for h in (1, 2, 7, 90, 1080):
        for n in (1, 2, 3, 7, 8):
            rows = [r for k in range(n) for r in range(*split_rows(h, n, k)[:2])]
            assert rows == list(range(h)), (h, n)
            assert len({split_rows(h, n, k)[2] for k in range(n)}) == 1


def _gather_rank(rank, world_size, port, q, W, H):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world_size))
    import torch
    import torch.distributed as dist

    from voxelg_b200.replicas import gather_rows, split_rows
    dist.init_process_group("gloo", rank=rank, world_size=world_size,
                            timeout=timedelta(seconds=60))
    try:
        y0, y1, per = split_rows(H, world_size, rank)
        rec = torch.zeros(world_size * per * W * 24, dtype=torch.uint8)
        sh = torch.zeros(world_size * per * W * 8, dtype=torch.uint8)
        for y in range(y0, y1):          # this rank's rows, as the row renderer writes them
            rec[y * W * 24:(y + 1) * W * 24] = (y * 7 + 1) % 251
            sh[y * W * 8:(y + 1) * W * 8] = (y * 3 + 2) % 253
        got_rec, got_sh = gather_rows(rec, sh, W, H)
        q.put((rank, got_rec.numpy().tobytes(), got_sh.numpy().tobytes()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_a_frame_split_by_rows():
    import torch.multiprocessing as mp
    W, H = 5, 7                          # odd: the last rank's slice has a padding row
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, q, W, H)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    want_rec = b"".join(bytes([(y * 7 + 1) % 251]) * (W * 24) for y in range(H))
    want_sh = b"".join(bytes([(y * 3 + 2) % 253]) * (W * 8) for y in range(H))
    for _, rec, sh in got:
        assert rec == want_rec and sh == want_sh


@pytest.mark.gpu
def test_row_ranges_compose_the_frame():
    """vx_render_primary_rows: uneven row ranges rendered into one buffer give
    the whole frame's records; rows outside a range stay untouched; a range
    past the frame is rejected."""
    import torch

    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    cam = vg.default_camera(dw, 160, 90)
    p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM | po.OR_F_SHADOW)
    whole, whole_sh = vg.render_primary(dw, cam, p)
    rec = torch.full_like(whole, 0xAB)
    sh = torch.full_like(whole_sh, 0xCD)
    vg.render_primary_rows(dw, cam, p, 37, 38, rec, sh)
    torch.cuda.synchronize()
    r, s = rec.cpu().numpy(), sh.cpu().numpy()
    assert np.array_equal(r[37 * 160 * 24:38 * 160 * 24], whole.cpu().numpy()[37 * 160 * 24:38 * 160 * 24])
    assert (r[:37 * 160 * 24] == 0xAB).all() and (r[38 * 160 * 24:] == 0xAB).all()
    assert (s[:37 * 160 * 8] == 0xCD).all() and (s[38 * 160 * 8:] == 0xCD).all()
    for y0, y1 in ((0, 37), (38, 90), (90, 90)):
        vg.render_primary_rows(dw, cam, p, y0, y1, rec, sh)
    torch.cuda.synchronize()
    assert np.array_equal(rec.cpu().numpy(), whole.cpu().numpy())
    assert np.array_equal(sh.cpu().numpy(), whole_sh.cpu().numpy())
    big = torch.empty(91 * 160 * 24, dtype=torch.uint8, device=rec.device)
    with pytest.raises(L.VxError):                  # the library rejects rows past the frame
        vg.render_primary_rows(dw, cam, p, 10, 91, big, None)
    with pytest.raises(ValueError):                 # the binding rejects short buffers
        vg.render_primary_rows(dw, cam, p, 0, 90, rec[:100], sh)
    dw.close()


@pytest.mark.gpu
def test_nccl_split_frame_equals_the_frame():
    """render_split over one NCCL rank: the row slices travel through the
    all-gather and assemble the frame of vx_render_primary."""
    import torch
    import torch.distributed as dist

    import voxelg_b200 as vg
    from voxelg_b200.replicas import render_split
    torch.cuda.set_device(0)
    port = _free_port()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                            world_size=1, timeout=timedelta(seconds=60))
    try:
        cfg = vg.CONFIGS["c1"]
        dw = vg.DeviceWorld(*cfg.bricks)
        dw.generate(cfg.terrain)
        cam = vg.default_camera(dw, 200, 113)
        p = vg.default_params(po.OR_F_L4 | po.OR_F_LUT | po.OR_F_LOD | po.OR_F_BEAM | po.OR_F_SHADOW)
        rec, sh = render_split(dw, cam, p)
        whole, whole_sh = vg.render_primary(dw, cam, p)
        torch.cuda.synchronize()
        assert np.array_equal(rec.cpu().numpy(), whole.cpu().numpy())
        assert np.array_equal(sh.cpu().numpy(), whole_sh.cpu().numpy())
        dw.close()
    finally:
        dist.destroy_process_group()
