"""Ray-query messages in voxelG's network framing (vx_wire_* in
include/voxrt.h): RayQuery / RayResult frames that clients of src/net.rs
exchange with the serving loop."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def encode_query(qid: int, rays: np.ndarray) -> bytes:
    rays = np.ascontiguousarray(rays).view(L.RAY_DTYPE)
    lib = L.load()
    n = len(rays)
    buf = np.empty(lib.vx_wire_query_bytes(n), np.uint8)
    out = C.c_size_t()
    L.check(lib.vx_wire_encode_query(qid, C.c_void_p(rays.ctypes.data if n else 0), n,
                                     C.c_void_p(buf.ctypes.data), buf.size, C.byref(out)))
    return buf[: out.value].tobytes()


def decode_query(frame: bytes):
    """(id, RAY_DTYPE array) of a RayQuery frame."""
    lib = L.load()
    raw = np.frombuffer(frame, np.uint8)
    cap = max(0, (len(frame) - 24) // 32)
    rays = np.zeros(cap, L.RAY_DTYPE)
    qid, n = C.c_uint64(), C.c_size_t()
    L.check(lib.vx_wire_decode_query(C.c_void_p(raw.ctypes.data), len(frame), C.byref(qid),
                                     C.c_void_p(rays.ctypes.data if cap else 0), cap,
                                     C.byref(n)))
    return int(qid.value), rays[: n.value]


def encode_result(qid: int, records: np.ndarray) -> bytes:
    rec = np.ascontiguousarray(records).view(L.RECORD_DTYPE)
    lib = L.load()
    n = len(rec)
    buf = np.empty(lib.vx_wire_result_bytes(n), np.uint8)
    out = C.c_size_t()
    L.check(lib.vx_wire_encode_result(qid, C.c_void_p(rec.ctypes.data if n else 0), n,
                                      C.c_void_p(buf.ctypes.data), buf.size, C.byref(out)))
    return buf[: out.value].tobytes()


def decode_result(frame: bytes):
    """(id, RECORD_DTYPE array) of a RayResult frame."""
    lib = L.load()
    raw = np.frombuffer(frame, np.uint8)
    cap = max(0, (len(frame) - 24) // 23)
    rec = np.zeros(cap, L.RECORD_DTYPE)
    qid, n = C.c_uint64(), C.c_size_t()
    L.check(lib.vx_wire_decode_result(C.c_void_p(raw.ctypes.data), len(frame), C.byref(qid),
                                      C.c_void_p(rec.ctypes.data if cap else 0), cap,
                                      C.byref(n)))
    return int(qid.value), rec[: n.value]
