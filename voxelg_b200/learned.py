"""The learned start-distance proposal (vx_proposal_* / vx_render_learned in
include/voxrt.h): an MLP trained on the device on rays labelled by the plain
DDA, whose per-ray proposal bounds a verification walk after which the DDA
restarts.  Records equal the plain DDA's except `steps`."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .world import DeviceWorld


def default_config(**overrides) -> L.VxTrainConfig:
    c = L.VxTrainConfig()
    L.check(L.load().vx_proposal_default_config(C.byref(c)))
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


@dataclass
class FrameStats:
    none: int
    partial: int
    accepted: int
    miss: int
    cells: int
    iters: int
    fallback: int
    rays: int
    infer_ms: float
    trace_ms: float

    @property
    def acceptance(self) -> float:
        return self.accepted / max(self.rays, 1)


def _stats(s: L.VxLearnedStats) -> FrameStats:
    return FrameStats(int(s.none), int(s.partial), int(s.accepted), int(s.miss), int(s.cells),
                      int(s.iters), int(s.fallback), int(s.rays), float(s.infer_ms),
                      float(s.trace_ms))


class Proposal:
    """MLP parameters + Adam state on the world's device."""

    def __init__(self, world: DeviceWorld, seed: int = 1):
        self._lib = L.load()
        self.device = world.device
        h = C.c_void_p()
        L.check(self._lib.vx_proposal_create(world.handle, C.c_uint64(seed), C.byref(h)))
        self.handle = h

    # parameters -----------------------------------------------------------
    def params(self) -> np.ndarray:
        out = np.empty(L.MLP_FLOATS, np.float32)
        L.check(self._lib.vx_proposal_get_params(self.handle, C.c_void_p(out.ctypes.data),
                                                 out.size))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        L.check(self._lib.vx_proposal_set_params(self.handle, C.c_void_p(p.ctypes.data), p.size))

    # building blocks ------------------------------------------------------
    def features(self, world: DeviceWorld, rays, origin=(0, 0, 0)):
        """Features (n x 80 float32 CUDA tensor) of rays (numpy RAY array or
        CUDA uint8 tensor)."""
        import torch
        dev = torch.device("cuda", self.device)
        if isinstance(rays, np.ndarray):
            rays = torch.from_numpy(np.ascontiguousarray(rays).view(np.uint8).reshape(-1)).to(dev)
        n = rays.numel() // 32
        f = torch.empty((n, L.MLP_FEATURES), dtype=torch.float32, device=dev)
        L.check(self._lib.vx_proposal_features(self.handle, world.handle, L.i3(origin),
                                               C.c_void_p(rays.data_ptr()), n,
                                               C.c_void_p(f.data_ptr()), None))
        torch.cuda.synchronize(dev)
        return f

    def grad(self, feats, targets):
        """(loss, gradient[MLP_FLOATS]) of the FP32 forward/backward kernels."""
        g = np.empty(L.MLP_FLOATS, np.float32)
        loss = C.c_float()
        n = int(feats.shape[0])
        L.check(self._lib.vx_proposal_grad(self.handle, C.c_void_p(feats.data_ptr()),
                                           C.c_void_p(targets.data_ptr()), n,
                                           C.c_void_p(g.ctypes.data), C.byref(loss)))
        return float(loss.value), g

    def infer(self, feats):
        """BF16 tensor-core inference: predicted log t per row (CUDA tensor)."""
        import torch
        n = int(feats.shape[0])
        out = torch.empty(n, dtype=torch.float32, device=feats.device)
        L.check(self._lib.vx_proposal_infer(self.handle, C.c_void_p(feats.data_ptr()), n,
                                            C.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize(feats.device)
        return out

    def train(self, world: DeviceWorld, config: L.VxTrainConfig | None = None):
        """Label rays of random poses with the plain DDA and train; returns
        (loss curve, held-out loss before, after)."""
        c = config or default_config()
        curve = np.zeros(max(int(c.steps), 1), np.float32)
        held = (C.c_float * 2)()
        L.check(self._lib.vx_proposal_train(self.handle, world.handle, C.byref(c),
                                            C.c_void_p(curve.ctypes.data), held))
        return curve[: int(c.steps)], float(held[0]), float(held[1])

    def close(self):
        if getattr(self, "handle", None):
            self._lib.vx_proposal_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_learned(world: DeviceWorld, proposal: Proposal | None, cam: L.VxCamera,
                   params: L.VxTraceParams, rec, scale: float = 1.0, stats: bool = True,
                   stream: int = 0):
    """Learned-form primary frame into rec (CUDA uint8 tensor, 24 B/pixel).
    proposal None = verify until the walk fails.  Returns FrameStats (or None
    with stats=False, asynchronous on `stream`)."""
    s = L.VxLearnedStats()
    L.check(L.load().vx_render_learned(world.handle, proposal.handle if proposal else None,
                                       C.byref(cam), C.byref(params), C.c_float(scale),
                                       C.c_void_p(rec.data_ptr()),
                                       C.byref(s) if stats else None, C.c_void_p(stream)))
    return _stats(s) if stats else None
