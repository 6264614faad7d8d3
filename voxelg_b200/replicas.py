"""World replicas across ranks, one process per GPU.

Rays are independent and the world is read-only within a frame, so every rank
holds the whole world on its own device and traces its own rays with no
exchange.  The one exchange is an edit: the dirty bricks that the editing
rank's world changed (the upload set of voxelG's Renderer::upload_world,
src/renderer.rs:1345-1394) go to every rank before the next frame, and each
rank applies them to its replica with vx_world_apply_dirty.

broadcast_dirty does that over torch.distributed: NCCL broadcasts from device
buffers, gloo from host buffers.  Every rank calls it the same number of
times in the same order, as every collective requires.
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
