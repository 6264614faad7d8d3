"""World replicas across ranks, one process per GPU.

Rays are independent and the world is read-only within a frame, so every rank
holds the whole world on its own device and traces its own rays.  Two
exchanges remain:
- an edit: the dirty bricks that the editing rank's world changed (the upload
  set of voxelG's Renderer::upload_world, src/renderer.rs:1345-1394) go to
  every rank before the next frame, and each rank applies them to its replica
  with vx_world_apply_dirty (broadcast_dirty);
- one frame split across ranks by rows: each rank traces its range of rows
  (vx_render_primary_rows) and the ranges are gathered into the whole frame
  on every rank (render_split).

Both run over torch.distributed: NCCL from device buffers, gloo from host
buffers.  Every rank calls them the same number of times in the same order,
as every collective requires.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from . import _lib as L

BRICK_BYTES = L.BRICK_DTYPE.itemsize


def broadcast_dirty(world=None, brick_idx: Optional[np.ndarray] = None,
                    bricks: Optional[np.ndarray] = None, src: int = 0, group=None,
                    apply: Optional[Callable[[np.ndarray, np.ndarray], None]] = None,
                    stream: int = 0):
    """Send rank `src`'s dirty set (brick indices and their 72-byte bricks)
    to every rank of `group` and apply it to each rank's replica.

    On `src`, brick_idx and bricks hold the set (duplicates allowed: the
    last occurrence wins when it is applied); elsewhere they are ignored.
    `world` is this rank's DeviceWorld (vx_world_apply_dirty on `stream`);
    `apply(idx, bricks)` replaces that step for other replicas.  Returns the
    (idx, bricks) every rank received; the same arrays on every rank."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank()
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        dev = torch.device("cpu")
    n_t = torch.zeros(1, dtype=torch.int64, device=dev)
    if rank == src:
        idx = np.ascontiguousarray(brick_idx, dtype=np.uint32).reshape(-1)
        b = np.ascontiguousarray(bricks).view(L.BRICK_DTYPE).reshape(-1)
        if len(idx) != len(b):
            raise ValueError("broadcast_dirty: brick_idx and bricks differ in length")
        n_t[0] = len(idx)
    dist.broadcast(n_t, src, group=group)
    n = int(n_t.item())
    if n == 0:
        return np.zeros(0, np.uint32), np.zeros(0, L.BRICK_DTYPE)
    idx_t = torch.empty(n, dtype=torch.int32, device=dev)
    b_t = torch.empty(n * BRICK_BYTES, dtype=torch.uint8, device=dev)
    if rank == src:
        idx_t.copy_(torch.from_numpy(idx.view(np.int32)))
        b_t.copy_(torch.from_numpy(b.view(np.uint8)))
    dist.broadcast(idx_t, src, group=group)
    dist.broadcast(b_t, src, group=group)
    got_idx = idx_t.cpu().numpy().view(np.uint32)
    got_b = b_t.cpu().numpy().view(L.BRICK_DTYPE)
    if apply is not None:
        apply(got_idx, got_b)
    elif world is not None:
        world.apply_dirty(got_idx, got_b, stream)
    return got_idx, got_b


def split_rows(height: int, ranks: int, rank: int) -> tuple[int, int, int]:
    """Rows of a `height`-row frame for `rank` of `ranks`: (y0, y1, rows per
    rank).  Every rank owns the same number of row slots, rows_per = ceil(
    height / ranks), so that the gather moves equal slices; the slots past
    the frame's last row stay empty."""
    per = -(-int(height) // int(ranks))
    y0 = min(int(height), rank * per)
    return y0, min(int(height), y0 + per), per


def gather_rows(rec, shadow, width: int, height: int, group=None):
    """All-gather the row slices of a frame split by split_rows: rank r
    contributes rows [r * per, (r + 1) * per) of its frame-sized buffers (24
    and 8 bytes a record, rows past the frame's end included as padding).
    Returns the whole frame's (records, shadows) as uint8 tensors on every
    rank, in the buffers' device; shadow may be None."""
    import torch
    import torch.distributed as dist

    ranks = dist.get_world_size(group)
    rank = dist.get_rank(group)
    _, _, per = split_rows(height, ranks, rank)
    out = []
    for buf, size in ((rec, 24), (shadow, 8)):
        if buf is None:
            out.append(None)
            continue
        row = int(width) * size
        if buf.numel() < ranks * per * row:
            raise ValueError("gather_rows: buffers must hold ranks * rows_per rows")
        full = torch.empty(ranks * per * row, dtype=torch.uint8, device=buf.device)
        mine = buf[rank * per * row:(rank + 1) * per * row]
        dist.all_gather_into_tensor(full, mine, group=group)
        out.append(full[:int(height) * row])
    return out[0], out[1]


def render_split(world, cam, params, group=None, stream: int = 0):
    """One frame split across the ranks of `group` by rows: each rank traces
    its rows (vx_render_primary_rows) on its own replica of the world and the
    row ranges are all-gathered.  Returns the whole frame's (records,
    shadows) uint8 CUDA tensors on every rank; they equal vx_render_primary's
    frame.  Call it with the same camera and parameters on every rank."""
    import torch
    import torch.distributed as dist

    from .trace import render_primary_rows

    ranks = dist.get_world_size(group)
    rank = dist.get_rank(group)
    W, H = int(cam.res_x), int(cam.res_y)
    y0, y1, per = split_rows(H, ranks, rank)
    dev = torch.device("cuda", world.device)
    rec = torch.zeros(ranks * per * W * 24, dtype=torch.uint8, device=dev)
    shadow = None
    if params.flags & L.VX_F_SHADOW:
        shadow = torch.zeros(ranks * per * W * 8, dtype=torch.uint8, device=dev)
    render_primary_rows(world, cam, params, y0, y1, rec, shadow, stream)
    torch.cuda.synchronize(dev)
    return gather_rows(rec, shadow, W, H, group)
