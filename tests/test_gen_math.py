"""The chunk generator's powf / cosf / sinf against the host C library.

The reference's generator calls f32::powf (src/voxel.rs:1262 mountain
height, :1623 pine canopy radius) and f32::cos / f32::sin (:1639-1641,
:1695-1697 branch ends): on Linux, glibc's powf, cosf and sinf.  The
library reproduces them (voxelg_b200/csrc/vx_gmath.h) and must return the
same binary32 bits on the generator's domains: every float x in [0, 1] for
powf(x, 1.15f) and powf(x, 0.85f), and every branch angle paint_tree can
form for cosf and sinf.  The checker is glibc itself (oracle or_libm_batch).

- CPU: the exception table was built against the C library this process
  runs; the host evaluation equals glibc on every branch angle and on every
  64th float of [0, 1] plus every tabled input.
- GPU: the device evaluation equals glibc on every float of [0, 1] for both
  exponents (1,065,353,217 inputs each) and on every branch angle.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from voxelg_b200 import _lib as L

POW115, POW085, COS, SIN = 0, 1, 2, 3
ONE_BITS = 0x3F800000  # 1.0f


def branch_angles():
    """Every angle of src/voxel.rs:1633-1634 / :1689-1690: branch b of n (2-3
    for birch with spread 0.5, 3-4 for oak and autumn with spread 0.6) at
    each of the 65536 jitter values, in binary32 in the reference's order."""
    f = np.float32
    j = np.arange(65536, dtype=np.float32)
    jit = (j / f(65535.0)) * f(2.0) - f(1.0)
    tau = f(6.28318548202514648)
    out = []
    for ns, spread in (((2, 3), f(0.5)), ((3, 4), f(0.6))):
        for n in ns:
            for b in range(n):
                out.append((f(b) / f(n)) * tau + jit * spread)
    return np.unique(np.concatenate(out).astype(np.float32))


def host_math(fn, x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    L.check(L.load().vx_gen_math_host(fn, C.c_void_p(x.ctypes.data), len(x),
                                      C.c_void_p(out.ctypes.data)))
    return out


def table_path():
    return L.LIB_PATH.parent / "vx_libm_exceptions.bin"


def test_table_was_built_for_this_c_library():
    blob = np.fromfile(table_path(), dtype="<u4")
    assert blob[0] == 0x4D4C5856 and blob[1] == 1 and blob[10] == 4
    ver = blob[2:10].tobytes().split(b"\0")[0].decode()
    libc = C.CDLL("libc.so.6")
    libc.gnu_get_libc_version.restype = C.c_char_p
    assert ver == libc.gnu_get_libc_version().decode()


def tabled_inputs(fn):
    blob = np.fromfile(table_path(), dtype="<u4")
    off = int(blob[11 + fn])
    n = int(blob[off])
    keys = blob[off + 1 + 65537: off + 1 + 65537 + n]
    assert np.all(np.diff(keys.astype(np.int64)) > 0)
    return keys


@pytest.mark.parametrize("fn", [POW115, POW085])
def test_host_pow_equals_glibc(fn):
    bits = np.concatenate([np.arange(0, ONE_BITS + 1, 64, dtype=np.uint32),
                           tabled_inputs(fn), np.array([ONE_BITS], np.uint32)])
    x = bits.view(np.float32)
    got, want = host_math(fn, x), po.libm_batch(fn, x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the table is needed: without it the library's own evaluation differs
    assert len(tabled_inputs(fn)) > 100000


@pytest.mark.parametrize("fn", [COS, SIN])
def test_host_trig_equals_glibc_on_every_branch_angle(fn):
    a = branch_angles()
    assert 600000 < len(a) < 800000
    got, want = host_math(fn, a), po.libm_batch(fn, a)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_gen_math_arguments():
    x = np.zeros(4, np.float32)
    assert L.load().vx_gen_math_host(7, C.c_void_p(x.ctypes.data), 4,
                                     C.c_void_p(x.ctypes.data)) == L.VX_ERR_INVALID
    assert L.load().vx_gen_math_host(0, None, 0, None) == 0


@pytest.mark.gpu
def test_device_math_equals_glibc_exhaustively():
    """Every float of [0, 1] for both exponents, and every branch angle, on
    the device, bit for bit against glibc on this host."""
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    import voxelg_b200 as vg
    dw = vg.DeviceWorld(64, 16, 64)
    lib = L.load()
    threads = os.cpu_count() or 1
    chunk = 1 << 26
    try:
        xin = torch.empty(chunk, dtype=torch.float32, device="cuda")
        xout = torch.empty(chunk, dtype=torch.float32, device="cuda")
        # torch writes the inputs on its stream; the library's calls (stream
        # NULL = the world's own stream, waited for) start after a device sync
        stream = None
        for fn in (POW115, POW085):
            bad = 0
            for start in range(0, ONE_BITS + 1, chunk):
                n = min(chunk, ONE_BITS + 1 - start)
                bits = torch.arange(start, start + n, dtype=torch.int64, device="cuda")
                xin[:n] = bits.to(torch.int32).view(torch.float32)
                torch.cuda.synchronize()
                L.check(lib.vx_gen_math(dw.handle, fn, C.c_void_p(xin.data_ptr()), n,
                                        C.c_void_p(xout.data_ptr()), stream))
                got = xout[:n].cpu().numpy().view(np.uint32)
                want = po.libm_batch(fn, xin[:n].cpu().numpy(), threads).view(np.uint32)
                bad += int(np.count_nonzero(got != want))
            assert bad == 0, (fn, bad)
        a = branch_angles()
        t = torch.from_numpy(a).cuda()
        out = torch.empty_like(t)
        torch.cuda.synchronize()
        for fn in (COS, SIN):
            L.check(lib.vx_gen_math(dw.handle, fn, C.c_void_p(t.data_ptr()), len(a),
                                    C.c_void_p(out.data_ptr()), stream))
            got = out.cpu().numpy().view(np.uint32)
            want = po.libm_batch(fn, a, threads).view(np.uint32)
            assert np.array_equal(got, want), fn
    finally:
        dw.close()
