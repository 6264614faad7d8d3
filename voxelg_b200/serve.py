"""Ray-query serving loop with continuous batching over device slots, or as
a device-resident request loop (vx_server_* in include/voxrt.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .world import DeviceWorld


def stats_dict(st: L.VxServeStats) -> dict:
    return {k: getattr(st, k) for k, _ in L.VxServeStats._fields_}


class Server:
    """Ray-query server over a DeviceWorld (which must outlive it)."""

    def __init__(self, world: DeviceWorld, params: L.VxTraceParams, origin=(0, 0, 0),
                 mem_budget_bytes: int = 256 << 20, slots: int = 4, max_batch_rays: int = 0,
                 max_batch_requests: int = 0, resident: bool = False, idle_us: int = 0,
                 wait_us: int = 0):
        """resident=True runs the device-resident request loop
        (VX_SERVE_RESIDENT); slots and max_batch_requests then do not apply."""
        self._lib = L.load()
        self.world = world
        mode = L.VX_SERVE_RESIDENT if resident else L.VX_SERVE_SLOTS
        cfg = L.VxServeConfig(mem_budget_bytes, slots, max_batch_rays, max_batch_requests, mode,
                              idle_us, wait_us)
        h = C.c_void_p()
        L.check(self._lib.vx_server_create(world.handle, L.i3(origin), C.byref(params),
                                           C.byref(cfg), C.byref(h)))
        self.handle = h
        self._live = {}

    def submit(self, rays: np.ndarray, out: np.ndarray | None = None) -> int:
        """Queue rays (RAY_DTYPE); returns a ticket.  The result array (a new
        one, or `out` of RECORD_DTYPE and len(rays)) is held by the server
        object until collected with wait().  Arrays in page-locked memory
        are read and written in place by the resident loop."""
        rays = np.ascontiguousarray(rays).view(L.RAY_DTYPE)
        if out is None:
            out = np.zeros(len(rays), L.RECORD_DTYPE)
        elif out.dtype != L.RECORD_DTYPE or len(out) != len(rays) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous RECORD_DTYPE array of len(rays)")
        t = C.c_uint64()
        L.check(self._lib.vx_server_submit(self.handle, C.c_void_p(L.ptr(rays)), len(rays),
                                           C.c_void_p(L.ptr(out)), C.byref(t)))
        self._live[t.value] = (rays, out)
        return t.value

    def wait(self, ticket: int, timeout_s: float = 30.0) -> np.ndarray:
        rc = L.check(self._lib.vx_server_wait(self.handle, ticket, timeout_s))
        if rc != 1:
            raise TimeoutError(f"request {ticket} not done after {timeout_s} s")
        return self._live.pop(ticket)[1]

    def edit(self, brick_idx, bricks):
        idx = np.ascontiguousarray(brick_idx, dtype=np.uint32)
        b = np.ascontiguousarray(bricks).view(L.BRICK_DTYPE)
        L.check(self._lib.vx_server_edit(self.handle, C.c_void_p(L.ptr(idx)),
                                         C.c_void_p(L.ptr(b)), len(idx)))

    def stats(self, reset: bool = False) -> dict:
        st = L.VxServeStats()
        L.check(self._lib.vx_server_stats(self.handle, C.byref(st), 1 if reset else 0))
        return stats_dict(st)

    def bench(self, clients=64, rate_per_client=200.0, seconds=5.0, min_rays=1, max_rays=50000,
              min_len=8.0, max_len=512.0, edit_fraction_per_s=0.01, seed=1) -> dict:
        load = L.VxServeLoad(clients, rate_per_client, seconds, min_rays, max_rays, min_len,
                             max_len, edit_fraction_per_s, seed)
        st = L.VxServeStats()
        L.check(self._lib.vx_serve_bench(self.handle, C.byref(load), C.byref(st)))
        return stats_dict(st)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.vx_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
