"""Ray-query messages in voxelG's network framing (src/net.rs:46-90): the C
codec against an independent restatement of bincode 1.3.3's default
encoding, malformed frames, and a query served end to end through the
serving loop."""
import struct

import numpy as np
import pytest

from oracle import pyoracle as po


def bincode_query(qid, rays):
    """net.rs write_message of Message::RayQuery (variant 10) as bincode 1.x
    writes it: u32 variant, u64 fields, Vec as u64 count + elements, f32 /
    u32 little-endian, fixed arrays inline."""
    body = struct.pack("<IQQ", 10, qid, len(rays))
    for r in rays:
        body += struct.pack("<7fI", *r["org"], *r["dir"], r["tmax"], r["kind"])
    return struct.pack("<I", len(body)) + body


def bincode_result(qid, rec):
    body = struct.pack("<IQQ", 11, qid, len(rec))
    for r in rec:
        body += struct.pack("<3iBBBfI", *r["voxel"], r["face"], r["mat"], r["flags"], r["t"],
                            r["steps"])
    return struct.pack("<I", len(body)) + body


def _rays(n, seed=0):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, po.RAY)
    r["org"] = rng.uniform(-1e3, 1e3, (n, 3)).astype(np.float32)
    r["dir"] = rng.normal(size=(n, 3)).astype(np.float32)
    r["tmax"] = rng.uniform(0, 700, n).astype(np.float32)
    r["kind"] = rng.integers(0, 3, n) | (rng.integers(0, 2, n) << 8)
    return r


def _records(n, seed=1):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, po.RECORD)
    r["voxel"] = rng.integers(-2**31, 2**31 - 1, (n, 3))
    r["face"] = rng.integers(0, 256, n)
    r["mat"] = rng.integers(0, 256, n)
    r["flags"] = rng.integers(0, 4, n)
    r["t"] = rng.uniform(0, 700, n).astype(np.float32)
    r["steps"] = rng.integers(0, 2**32 - 1, n, dtype=np.uint64)
    return r


@pytest.mark.parametrize("n", [0, 1, 7, 1000])
def test_query_bytes_are_bincode(n):
    from voxelg_b200 import wire
    rays = _rays(n)
    frame = wire.encode_query(0xDEADBEEF12345678, rays)
    assert frame == bincode_query(0xDEADBEEF12345678, rays)
    qid, back = wire.decode_query(frame)
    assert qid == 0xDEADBEEF12345678
    assert np.array_equal(back.view(np.uint8), rays.view(np.uint8))


@pytest.mark.parametrize("n", [0, 3, 500])
def test_result_bytes_are_bincode(n):
    from voxelg_b200 import wire
    rec = _records(n)
    frame = wire.encode_result(42, rec)
    assert frame == bincode_result(42, rec)
    qid, back = wire.decode_result(frame)
    assert qid == 42
    want = rec.copy()
    want["pad"] = 0
    assert np.array_equal(back.view(np.uint8), want.view(np.uint8))


def test_malformed_frames_are_rejected():
    from voxelg_b200 import _lib as L
    from voxelg_b200 import wire
    good = wire.encode_query(1, _rays(4))
    bad = [
        good[:10],                                            # shorter than the header
        good[:-1],                                            # length disagrees with prefix
        struct.pack("<I", len(good) - 3) + good[4:] + b"x",   # prefix off by one
        good[:4] + struct.pack("<I", 11) + good[8:],          # wrong variant
        good[:16] + struct.pack("<Q", 5) + good[24:],         # count disagrees with length
        struct.pack("<I", 16 * 1024 * 1024 + 1) + good[4:],   # over the 16 MiB limit
    ]
    for frame in bad:
        with pytest.raises(L.VxError) as e:
            wire.decode_query(frame)
        assert e.value.code == L.VX_ERR_INVALID
    with pytest.raises(L.VxError):
        wire.decode_result(good)                              # a query is not a result
    # a query too large for one frame is refused at encoding
    lib = L.load()
    assert lib.vx_wire_query_bytes(600_000) - 4 > 16 * 1024 * 1024


@pytest.mark.gpu
@pytest.mark.parametrize("resident", [False, True], ids=["slots", "resident"])
def test_query_frame_served_end_to_end(c1_oracle_world, resident):
    """A RayQuery frame decoded, served by the ray-query server (device slots,
    or the device-resident request loop), and its RayResult frame equal to
    the oracle's records for the same rays."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU required for -m gpu tests")
    import voxelg_b200 as vg
    import voxelg_b200.serve as sv
    from voxelg_b200 import wire
    cfg = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*cfg.bricks)
    dw.generate(cfg.terrain)
    p = vg.default_params(vg._lib.VX_F_L4 | vg._lib.VX_F_LUT | vg._lib.VX_F_LOD)
    srv = sv.Server(dw, p, slots=2, resident=resident)
    rng = np.random.default_rng(5)
    rays = np.zeros(3000, po.RAY)
    rays["org"] = rng.uniform([0, 80, 0], [512, 200, 512], (3000, 3)).astype(np.float32)
    d = rng.normal(size=(3000, 3)).astype(np.float32)
    d /= np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
    rays["dir"] = d
    rays["tmax"] = 300.0
    rays["kind"] = rng.integers(0, 3, 3000)
    qid, got = wire.decode_query(wire.encode_query(77, rays))
    out = srv.wait(srv.submit(got))
    rid, rec = wire.decode_result(wire.encode_result(qid, out))
    want = po.trace_batch(c1_oracle_world, rays, p)[0]
    assert rid == 77 and np.array_equal(rec.view(np.uint8), want.view(np.uint8))
    srv.close()
    dw.close()
