"""Known-answer vectors for the traversal, computed without the oracle.

Writes tests/golden/traversal.json: crafted worlds (axis-aligned boxes of
one material each), rays and cameras, and the record every traversal entry
point must produce for them.  Nothing here imports the C oracle, the CUDA
library or numpy's float32 arithmetic.  The expected records come from three
computations that share no code with them:

1. An exact emulation of the reference traversal as the WGSL states it
   (shaders/raymarch.wgsl: dda_init :3369-3411, dda_step :3416-3448,
   trace :4600-4777, skip_to_cell :4807-4864, trace_no_water :3450-3532,
   trace_any :4345-4409 with shadow_voxel_occludes :4314-4343,
   entry_normal_and_t :3321-3342, brick_topmost_material :253-295,
   tile_representative_material :4782-4798, ray_dir_uv :430-438 and the
   pixel uv of cs_main :600) and of the CPU picking walk (src/raycast.rs:21-133).
   Every binary32 operation is evaluated on rationals (fractions.Fraction)
   and rounded to the nearest binary32, ties to even, as IEEE 754 defines
   it; sqrt is rounded the same way.  The world is a list of boxes: cell
   emptiness, brick and tile uniformity (src/voxel.rs:233-270) and the
   topmost / representative materials are read off the boxes, not off mask
   words.
2. Exact geometry: for every hit that resolves at a voxel (not a uniform or
   LOD early-out) the first opaque box the ray enters, its entry t, entry
   face and entry voxel follow from a slab test on rationals, with no
   traversal at all; the emulation must agree.  Early-out hits are checked
   to sit in a uniform (LUT) or non-empty (LOD) cell entered past the
   threshold, before any opaque voxel.
3. Hand-derived answers: a few rays whose whole record (including the
   iteration count) is worked out by hand in the comments of HAND below;
   the emulation must reproduce them.

The reference leaves a few points to the implementation; these vectors
avoid them rather than pin a choice: no value whose sign of zero reaches a
record, no float-to-int conversion out of the i32 range, and no voxel whose
reference resolution is a sub-voxel routine (foliage within
FOLIAGE_NEAR_T = 128, water within WATER_FAR_T = 400 for first hits;
decoration and leaves within 128 for any-hit rays).  The emulation raises
if a case reaches one of those, so every committed case is one where the
reference's own arithmetic, under IEEE binary32 without contraction, fixes
the record.

Usage: python tests/golden/make_golden.py   (rewrites traversal.json)
"""
from __future__ import annotations

import json
import math
import os
import sys
from fractions import Fraction as Q

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "traversal.json")

# ---------------------------------------------------------------- binary32

F32_MAX = (2 - Q(1, 2 ** 23)) * Q(2) ** 127


def rnd(q: Q) -> Q:
    """Nearest binary32 value to the rational q, ties to even."""
    q = Q(q)
    if q == 0:
        return Q(0)
    sign = -1 if q < 0 else 1
    a = -q if q < 0 else q
    n, d = a.numerator, a.denominator
    e = n.bit_length() - d.bit_length()
    if (n << max(0, -e)) < (d << max(0, e)):
        e -= 1                          # now 2^e <= a < 2^(e+1)
    ue = max(e, -126) - 23              # exponent of one unit in the last place
    num, den = (n, d << ue) if ue >= 0 else (n << -ue, d)
    m, r = divmod(num, den)
    if 2 * r > den or (2 * r == den and (m & 1)):
        m += 1
    v = Q(m) * (Q(2) ** ue)
    if v > F32_MAX:
        raise OverflowError("binary32 overflow")
    return sign * v


def lit(s: str) -> Q:
    """A WGSL / Rust f32 literal: the decimal rounded to binary32."""
    return rnd(Q(s))


def is_f32(q: Q) -> bool:
    return rnd(q) == q


def add(a, b):
    return rnd(a + b)


def sub(a, b):
    return rnd(a - b)


def mul(a, b):
    return rnd(a * b)


def div(a, b):
    return rnd(Q(a) / Q(b))


def _next_up(x: Q) -> Q:
    """Smallest binary32 above the positive binary32 x."""
    a = x
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if (a.numerator << max(0, -e)) < (a.denominator << max(0, e)):
        e -= 1
    return x + Q(2) ** (max(e, -126) - 23)


def _next_down(x: Q) -> Q:
    e = x.numerator.bit_length() - x.denominator.bit_length()
    if (x.numerator << max(0, -e)) < (x.denominator << max(0, e)):
        e -= 1
    ulp = Q(2) ** (max(e, -126) - 23)
    if x == Q(2) ** e and e > -126:
        ulp = ulp / 2                   # below a power of two the spacing halves
    return x - ulp


def fsqrt(x: Q) -> Q:
    """Correctly rounded binary32 square root of the binary32 x >= 0."""
    if x == 0:
        return Q(0)
    assert x > 0
    c = rnd(Q(math.sqrt(float(x))))    # a start within an ulp or two
    while True:
        up = _next_up(c)
        mid = (c + up) / 2
        if x > mid * mid or (x == mid * mid and _odd(c)):
            c = up
            continue
        dn = _next_down(c)
        mid = (dn + c) / 2
        if x < mid * mid or (x == mid * mid and _odd(c)):
            c = dn
            continue
        return c


def _odd(c: Q) -> bool:
    e = c.numerator.bit_length() - c.denominator.bit_length()
    if (c.numerator << max(0, -e)) < (c.denominator << max(0, e)):
        e -= 1
    m = c / Q(2) ** (max(e, -126) - 23)
    return int(m) & 1 == 1


def floor_i(q: Q) -> int:
    v = math.floor(q)
    if abs(v) >= 2 ** 30:
        raise ValueError("float-to-int conversion outside the range this suite pins")
    return v


def sgn(x: Q) -> int:
    return 1 if x > 0 else (-1 if x < 0 else 0)


def pos_mod(a: int, b: int) -> int:
    return a % b  # Python's % is the Euclidean remainder for b > 0 (common.wgsl:49-52)


EPS_INV = lit("1e-8")
BIG = lit("1e30")
BIAS = lit("1e-3")
EPS = lit("1e-6")
CLAMP = lit("0.01")


def safe_inv(x: Q) -> Q:
    """common.wgsl:55-58 / src/raycast.rs:139-141."""
    return BIG if abs(x) < EPS_INV else div(1, x)


# ---------------------------------------------------------------- materials
# shaders/raymarch.wgsl:875-920

STONE, DIRT, GRASS, GLASS, WATER, LEAVES, FLOWER, TALL_GRASS = 4, 3, 2, 18, 12, 14, 30, 31
LEAF_FRINGE, TURF, BUSH, SAND = 33, 35, 36, 1
FOLIAGE = {14, 25, 26, 27, 30, 31, 33, 34, 35, 36, 37}
DECORATION = {30, 31, 33, 34, 35, 36, 37}


def is_water(m):
    return 5 <= m <= 12


def is_transparent(m):
    return is_water(m) or m == GLASS


def uniform_optimisable(m):
    return m not in FOLIAGE and not is_transparent(m)


FOLIAGE_NEAR_T = Q(128)
WATER_FAR_T = Q(400)


class Deviation(Exception):
    """The case reaches a sub-voxel routine of the reference; not pinned."""


# ---------------------------------------------------------------- worlds


class Scene:
    """A window of bricks (bx, by, bz) at world voxel origin ro (ro.y = 0)
    holding non-overlapping boxes [x0, x1) x [y0, y1) x [z0, z1) given in
    world voxel coordinates inside the window, each of one material.  Slot
    space is the toroidal storage (raymarch.wgsl:17-23): x and z modulo the
    window size, y unchanged."""

    def __init__(self, name, bricks, ro, boxes):
        self.name = name
        self.bricks = tuple(bricks)
        self.V = tuple(4 * b for b in bricks)
        self.ro = tuple(ro)
        assert self.ro[1] == 0
        self.boxes = [tuple(b) for b in boxes]
        for b in self.boxes:
            assert b[6] != 0
            for k in range(3):
                assert self.ro[k] <= b[k] < b[k + 3] <= self.ro[k] + self.V[k], (name, b)
        for i, a in enumerate(self.boxes):
            for b in self.boxes[i + 1:]:
                assert not all(a[k] < b[k + 3] and b[k] < a[k + 3] for k in range(3)), (a, b)
        self.slot_boxes = []
        for b in self.boxes:
            for xs in self._split(b[0], b[3], self.V[0]):
                for zs in self._split(b[2], b[5], self.V[2]):
                    self.slot_boxes.append((xs[0], b[1], zs[0], xs[1], b[4], zs[1], b[6]))
        self._cache = {}

    @staticmethod
    def _split(a0, a1, n):
        s0 = a0 % n
        ln = a1 - a0
        if s0 + ln <= n:
            return [(s0, s0 + ln)]
        return [(s0, n), (0, s0 + ln - n)]

    def to_json(self):
        return {"name": self.name, "bricks": list(self.bricks), "origin": list(self.ro),
                "boxes": [list(b) for b in self.boxes]}

    # ---- slot-space queries
    def mat(self, s):
        for b in self.slot_boxes:
            if b[0] <= s[0] < b[3] and b[1] <= s[1] < b[4] and b[2] <= s[2] < b[5]:
                return b[6]
        return 0

    def empty(self, s, c):
        """Is the aligned slot cell of edge c holding slot voxel s empty?"""
        o = tuple(s[k] - s[k] % c for k in range(3))
        key = ("e", c, o)
        if key not in self._cache:
            self._cache[key] = not any(
                all(b[k] < o[k] + c and o[k] < b[k + 3] for k in range(3))
                for b in self.slot_boxes)
        return self._cache[key]

    def brick_uniform(self, s):
        """src/voxel.rs:233-247: fully solid, one nonzero material."""
        o = tuple(s[k] - s[k] % 4 for k in range(3))
        key = ("bu", o)
        if key not in self._cache:
            ms = {self.mat((o[0] + x, o[1] + y, o[2] + z))
                  for x in range(4) for y in range(4) for z in range(4)}
            self._cache[key] = ms.pop() if len(ms) == 1 and 0 not in ms else 0
        return self._cache[key]

    def tile_uniform(self, s):
        """src/voxel.rs:249-270: all 64 child bricks uniform, one material."""
        o = tuple(s[k] - s[k] % 16 for k in range(3))
        key = ("tu", o)
        if key not in self._cache:
            ms = {self.brick_uniform((o[0] + 4 * x, o[1] + 4 * y, o[2] + 4 * z))
                  for x in range(4) for y in range(4) for z in range(4)}
            self._cache[key] = ms.pop() if len(ms) == 1 and 0 not in ms else 0
        return self._cache[key]

    def brick_topmost(self, o):
        """raymarch.wgsl:253-295 for the brick at slot corner o: per layer
        y = 3..0, the voxel of lowest index x + 4z; turf is passed over."""
        any_occ = False
        for ly in (3, 2, 1, 0):
            for lz in range(4):
                hit = None
                for lx in range(4):
                    m = self.mat((o[0] + lx, o[1] + ly, o[2] + lz))
                    if m:
                        hit = m
                        break
                if hit is not None:
                    any_occ = True
                    if hit != TURF:
                        return hit
                    break
        return TURF if any_occ or self._occupied(o) else 0

    def _occupied(self, o):
        return not self.empty(o, 4)

    def tile_representative(self, s):
        """raymarch.wgsl:4782-4798: the first occupied child brick in the
        order x + 4z + 16y, then its topmost material."""
        o = tuple(s[k] - s[k] % 16 for k in range(3))
        for ly in range(4):
            for lz in range(4):
                for lx in range(4):
                    bo = (o[0] + 4 * lx, o[1] + 4 * ly, o[2] + 4 * lz)
                    if not self.empty(bo, 4):
                        return self.brick_topmost(bo)
        return 0


# ---------------------------------------------------------------- traversal

F_L4, F_LUT, F_LOD, F_BEAM = 1, 2, 4, 8
STOCK = F_L4 | F_LUT | F_LOD


class Params:
    def __init__(self, flags=STOCK, max_dist=700, lod_brick_t=400, tile_lod_t=520,
                 max_iters=1024, any_max_iters=768):
        self.flags = flags
        self.max_dist = lit(str(max_dist))
        self.lod_brick_t = lit(str(lod_brick_t))
        self.tile_lod_t = lit(str(tile_lod_t))
        self.max_iters = max_iters
        self.any_max_iters = any_max_iters

    def to_json(self):
        return {"flags": self.flags, "max_dist": float(self.max_dist),
                "lod_brick_t": float(self.lod_brick_t), "tile_lod_t": float(self.tile_lod_t),
                "max_iters": self.max_iters, "any_max_iters": self.any_max_iters}


class Walk:
    """The DDA state of dda_init / dda_step / skip_to_cell."""

    def __init__(self, sc: Scene, origin, d):
        self.sc = sc
        ro = sc.ro
        dims = [Q(v) for v in sc.V]
        self.d = d
        self.org = [sub(origin[k], Q(ro[k])) for k in range(3)]
        self.inv = [safe_inv(d[k]) for k in range(3)]
        t0 = [mul(-self.org[k], self.inv[k]) for k in range(3)]
        t1 = [mul(sub(dims[k], self.org[k]), self.inv[k]) for k in range(3)]
        self.tmin3 = [min(t0[k], t1[k]) for k in range(3)]
        tmax3 = [max(t0[k], t1[k]) for k in range(3)]
        self.t_enter = max(max(self.tmin3[0], self.tmin3[1]), max(self.tmin3[2], Q(0)))
        t_exit = min(min(tmax3[0], tmax3[1]), tmax3[2])
        self.valid = not (self.t_enter >= t_exit or t_exit < 0)
        if not self.valid:
            return
        self.step = [sgn(d[k]) for k in range(3)]
        self.tdel = [abs(v) for v in self.inv]
        te = add(self.t_enter, BIAS)
        vox = []
        for k in range(3):
            p = add(self.org[k], mul(d[k], te))
            p = min(max(p, CLAMP), sub(dims[k], CLAMP))
            vox.append(floor_i(p) + ro[k])
        self._set_voxel(vox)

    def _set_voxel(self, vox):
        ro = self.sc.ro
        self.voxel = list(vox)
        self.tmax = []
        for k in range(3):
            vl = vox[k] - ro[k]
            b = vl + 1 if self.step[k] > 0 else vl
            self.tmax.append(mul(sub(Q(b), self.org[k]), self.inv[k]))

    def slot(self):
        V = self.sc.V
        return (pos_mod(self.voxel[0], V[0]), self.voxel[1], pos_mod(self.voxel[2], V[2]))

    def in_window(self):
        return all(0 <= self.voxel[k] - self.sc.ro[k] < self.sc.V[k] for k in range(3))

    def step_once(self):
        tm = self.tmax
        if tm[0] < tm[1] and tm[0] < tm[2]:
            ax = 0
        elif tm[1] < tm[2]:
            ax = 1
        else:
            ax = 2
        t_cur = tm[ax]
        self.voxel[ax] += self.step[ax]
        tm[ax] = add(tm[ax], self.tdel[ax])
        return ax, t_cur

    def skip(self, cell):
        ro = self.sc.ro
        co = [self.voxel[k] - pos_mod(self.voxel[k], cell) for k in range(3)]
        tf = []
        for k in range(3):
            b = (co[k] + cell if self.step[k] > 0 else co[k]) - ro[k]
            tf.append(mul(sub(Q(b), self.org[k]), self.inv[k]))
        t_min, ax = BIG, 0
        for k in range(3):
            if self.step[k] != 0 and tf[k] > EPS and tf[k] < t_min:
                t_min, ax = tf[k], k
        if t_min == BIG:
            raise ValueError("skip without a forward face: outside what this suite pins")
        tb = add(t_min, BIAS)
        nv = [floor_i(add(self.org[k], mul(self.d[k], tb))) + ro[k] for k in range(3)]
        nv[ax] = co[ax] + cell if self.step[ax] > 0 else co[ax] - 1
        self._set_voxel(nv)
        return ax

    def entry(self, la):
        """entry_normal_and_t (raymarch.wgsl:3321-3342) as record fields."""
        if la >= 0:
            ax, t = la, sub(self.tmax[la], self.tdel[la])
        else:
            t = self.t_enter
            m = self.tmin3
            ax = 0 if (m[0] >= m[1] and m[0] >= m[2]) else (1 if m[1] >= m[2] else 2)
        return ax, t


def miss(steps):
    return {"voxel": [0, 0, 0], "face": 255, "mat": 0, "flags": 0, "t": Q(0), "steps": steps}


def hit_record(w: Walk, la, m, early, steps, **extra):
    ax, t = w.entry(la)
    if t == 0:
        raise ValueError("a zero t, whose sign the reference leaves open")
    r = {"voxel": list(w.voxel), "face": 2 * ax + (1 if w.step[ax] > 0 else 0), "mat": m,
         "flags": 1 | (2 if early else 0), "t": t, "steps": steps}
    r.update(extra)
    return r


def trace(sc: Scene, origin, d, max_dist, P: Params):
    """trace(), raymarch.wgsl:4600-4777, with the method switches F_*."""
    w = Walk(sc, origin, d)
    if not w.valid:
        return miss(0)
    la = -1
    t_cur = w.t_enter
    steps = 0
    for _ in range(P.max_iters):
        steps += 1
        if t_cur > max_dist or not w.in_window():
            return miss(steps)
        s = w.slot()
        cell = None
        if P.flags & F_L4:
            if sc.empty(s, 256):
                cell = 256
            elif sc.empty(s, 64):
                cell = 64
        if cell is None and sc.empty(s, 16):
            cell = 16
        if cell is not None:
            la = w.skip(cell)
            t_cur = sub(w.tmax[la], w.tdel[la])
            continue
        if P.flags & F_LOD and t_cur > P.tile_lod_t:
            lm = sc.tile_representative(s)
            if lm and uniform_optimisable(lm):
                return hit_record(w, la, lm, True, steps, why="tile LOD")
        if P.flags & F_LUT:
            tum = sc.tile_uniform(s)
            if tum and uniform_optimisable(tum):
                return hit_record(w, la, tum, True, steps, why="uniform tile")
        if sc.empty(s, 4):
            la = w.skip(4)
            t_cur = sub(w.tmax[la], w.tdel[la])
            continue
        if P.flags & F_LUT:
            bum = sc.brick_uniform(s)
            if bum and uniform_optimisable(bum):
                return hit_record(w, la, bum, True, steps, why="uniform brick")
        if P.flags & F_LOD and t_cur > P.lod_brick_t:
            m = sc.brick_topmost(tuple(s[k] - s[k] % 4 for k in range(3)))
            if m not in FOLIAGE:
                return hit_record(w, la, m, True, steps, why="brick LOD")
        m = sc.mat(s)
        if m:
            if m in FOLIAGE and t_cur <= FOLIAGE_NEAR_T:
                raise Deviation("near foliage")
            if is_water(m) and t_cur <= WATER_FAR_T:
                raise Deviation("near water")
            if m not in DECORATION:
                return hit_record(w, la, m, False, steps, why="voxel")
        la, t_cur = w.step_once()
    return miss(steps)


def trace_no_water(sc: Scene, origin, d, t_cap, P: Params):
    """trace_no_water, raymarch.wgsl:3450-3532: L4 always on, no uniform or
    LOD exits, transparent voxels passed, and t_cur moved only by dda_step."""
    w = Walk(sc, origin, d)
    if not w.valid:
        return miss(0)
    la = -1
    t_cur = w.t_enter
    steps = 0
    for _ in range(P.max_iters):
        steps += 1
        if t_cur > t_cap or not w.in_window():
            return miss(steps)
        s = w.slot()
        cell = 256 if sc.empty(s, 256) else (64 if sc.empty(s, 64) else (
            16 if sc.empty(s, 16) else (4 if sc.empty(s, 4) else None)))
        if cell is not None:
            la = w.skip(cell)
            continue
        m = sc.mat(s)
        if m and not is_transparent(m):
            return hit_record(w, la, m, False, steps, why="voxel")
        la, t_cur = w.step_once()
    return miss(steps)


def trace_any(sc: Scene, origin, d, max_dist, P: Params):
    """trace_any, raymarch.wgsl:4345-4409; record flags bit0 = occluded."""
    w = Walk(sc, origin, d)
    out = miss(0)
    if not w.valid:
        return out
    la = -1
    t_cur = w.t_enter
    steps = 0
    for _ in range(P.any_max_iters):
        steps += 1
        if t_cur > max_dist or not w.in_window():
            out["steps"] = steps
            return out
        s = w.slot()
        cell = 256 if sc.empty(s, 256) else (64 if sc.empty(s, 64) else (
            16 if sc.empty(s, 16) else (4 if sc.empty(s, 4) else None)))
        if cell is not None:
            la = w.skip(cell)
            t_cur = sub(w.tmax[la], w.tdel[la])
            continue
        m = sc.mat(s)
        if m:
            occ = True
            if m in (LEAF_FRINGE, TURF):
                occ = False
            elif m in DECORATION:
                if t_cur <= FOLIAGE_NEAR_T:
                    raise Deviation("near decoration on an any-hit ray")
                occ = False
            elif m in FOLIAGE and t_cur <= FOLIAGE_NEAR_T:
                raise Deviation("near leaves on an any-hit ray")
            if occ:
                out["flags"] = 1
                out["steps"] = steps
                return out
        la, t_cur = w.step_once()
    out["steps"] = steps
    return out


def run_kind(sc, origin, d, tmax, kind, P):
    if kind == 1:
        return trace_any(sc, origin, d, tmax, P)
    if kind == 2:
        return trace_no_water(sc, origin, d, tmax, P)
    return trace(sc, origin, d, tmax, P)


# ---------------------------------------------------------------- picking


def pick(sc: Scene, cam, d_in):
    """raycast(), src/raycast.rs:21-133, walking world coordinates."""
    dot = add(add(mul(d_in[0], d_in[0]), mul(d_in[1], d_in[1])), mul(d_in[2], d_in[2]))
    if dot == 0:
        return None
    rcp = div(1, fsqrt(dot))                     # glam normalize_or_zero
    d = [mul(v, rcp) for v in d_in]
    lo = [Q(sc.ro[k]) for k in range(3)]
    hi = [add(lo[k], Q(sc.V[k])) for k in range(3)]
    inv = [safe_inv(v) for v in d]
    t0 = [mul(sub(lo[k], cam[k]), inv[k]) for k in range(3)]
    t1 = [mul(sub(hi[k], cam[k]), inv[k]) for k in range(3)]
    tmn = [min(t0[k], t1[k]) for k in range(3)]
    tmx = [max(t0[k], t1[k]) for k in range(3)]
    t_enter = max(max(tmn), Q(0))
    t_exit = min(tmx)
    if t_enter >= t_exit or t_exit < 0:
        return None
    pb = lit("1e-3")
    te = add(t_enter, pb)
    p = [add(cam[k], mul(d[k], te)) for k in range(3)]
    p = [min(max(p[k], add(lo[k], pb)), sub(hi[k], pb)) for k in range(3)]
    voxel = [floor_i(v) for v in p]
    step = [sgn(v) for v in d]
    tdel = [abs(v) for v in inv]
    tmax = []
    for k in range(3):
        nxt = Q(voxel[k] + 1 if step[k] > 0 else voxel[k])
        tmax.append(mul(sub(nxt, cam[k]), inv[k]))

    def in_window(v):
        return all(0 <= v[k] - sc.ro[k] < sc.V[k] for k in range(3))

    def in_solid(v):
        if not in_window(v):
            return False
        s = (pos_mod(v[0], sc.V[0]), v[1], pos_mod(v[2], sc.V[2]))
        m = sc.mat(s)
        return m != 0 and m != LEAF_FRINGE

    def argmin_step():
        ax, m = -1, None
        for k in range(3):
            if step[k] != 0 and (m is None or tmax[k] < m):
                ax, m = k, tmax[k]
        if ax < 0:
            return -1
        voxel[ax] += step[ax]
        tmax[ax] = add(tmax[ax], tdel[ax])
        return ax

    last = -1
    left = 4096
    while left > 0 and in_solid(voxel):
        ax = argmin_step()
        if ax < 0:
            return None
        last = ax
        left -= 1
        if not in_window(voxel):
            return None
    while left > 0:
        if not in_window(voxel):
            return None
        if in_solid(voxel):
            n = [0, 0, 0]
            if last >= 0:
                n[last] = -step[last]
            return {"voxel": list(voxel), "normal": n}
        ax = argmin_step()
        if ax < 0:
            return None
        last = ax
        left -= 1
    return None


# ---------------------------------------------------------------- beam

BEAM_NONE = lit("1e9")
BEAM_MARGIN = Q(16)


def trunc_div(a: int, b: int) -> int:
    """WGSL i32 division (toward zero)."""
    q = abs(a) // b
    return q if a >= 0 else -q


def beam_first_tile(sc: Scene, origin, d):
    """trace_first_tile, beam.wgsl:51-113: a walk over 16-voxel tiles in
    world coordinates from the camera to the first tile whose bit is set in
    its chunk word; its entry t, or 1e9."""
    lo = [Q(sc.ro[k]) for k in range(3)]
    hi = [add(lo[k], Q(sc.V[k])) for k in range(3)]
    inv = [safe_inv(v) for v in d]
    t0 = [mul(sub(lo[k], origin[k]), inv[k]) for k in range(3)]
    t1 = [mul(sub(hi[k], origin[k]), inv[k]) for k in range(3)]
    tmn = [min(t0[k], t1[k]) for k in range(3)]
    tmx = [max(t0[k], t1[k]) for k in range(3)]
    t_enter = max(max(tmn[0], tmn[1]), max(tmn[2], Q(0)))
    t_exit = min(min(tmx[0], tmx[1]), tmx[2])
    if t_enter >= t_exit or t_exit < 0:
        return BEAM_NONE
    te = add(t_enter, lit("0.05"))
    c01 = lit("0.01")
    tile, step, tdel, tmax = [], [], [], []
    for k in range(3):
        p = add(origin[k], mul(d[k], te))
        p = min(max(p, add(lo[k], c01)), sub(hi[k], c01))
        tile.append(floor_i(div(p, 16)))
        step.append(sgn(d[k]))
        tdel.append(mul(abs(inv[k]), 16))
        b = (tile[k] + 1) * 16 if step[k] > 0 else tile[k] * 16
        tmax.append(mul(sub(Q(b), origin[k]), inv[k]))
    otile = [trunc_div(sc.ro[k], 16) for k in range(3)]
    T = [v // 16 for v in sc.V]
    t_cur = t_enter
    for _ in range(80):
        if not all(0 <= tile[k] - otile[k] < T[k] for k in range(3)):
            return BEAM_NONE
        st = (pos_mod(tile[0], T[0]), tile[1], pos_mod(tile[2], T[2]))
        if not sc.empty((16 * st[0], 16 * st[1], 16 * st[2]), 16):
            return t_cur
        if tmax[0] < tmax[1] and tmax[0] < tmax[2]:
            ax = 0
        elif tmax[1] < tmax[2]:
            ax = 1
        else:
            ax = 2
        tile[ax] += step[ax]
        t_cur = tmax[ax]
        tmax[ax] = add(tmax[ax], tdel[ax])
    return BEAM_NONE


def beam_pass(sc: Scene, cam):
    """cs_beam, beam.wgsl:30-49: one first-tile t per 8x8 pixel block."""
    bw, bh = (int(cam.res[0]) + 7) // 8, (int(cam.res[1]) + 7) // 8
    return [[beam_first_tile(sc, cam.origin, cam.beam_dir(gx, gy)) for gx in range(bw)]
            for gy in range(bh)]


# ---------------------------------------------------------------- cameras


class Camera:
    def __init__(self, origin, forward, right, up, tan_half_fov, res, jitter=(0, 0),
                 world_origin=(0, 0, 0)):
        self.origin = [Q(v) for v in origin]
        self.forward = [Q(v) for v in forward]
        self.right = [Q(v) for v in right]
        self.up = [Q(v) for v in up]
        self.tan = Q(tan_half_fov)
        self.res = (Q(res[0]), Q(res[1]))
        self.jitter = (Q(jitter[0]), Q(jitter[1]))
        self.world_origin = tuple(world_origin)
        for v in self.origin + self.forward + self.right + self.up + [self.tan]:
            assert is_f32(v)

    def ray_dir(self, px, py):
        """cs_main uv (raymarch.wgsl:600) and ray_dir_uv (:430-438)."""
        half = Q(1, 2)
        u = div(add(add(Q(px), half), self.jitter[0]), self.res[0])
        v = div(add(add(Q(py), half), self.jitter[1]), self.res[1])
        return self.dir_uv(u, v)

    def beam_dir(self, gx, gy):
        """cs_beam's ray through the centre of the 8x8 block (beam.wgsl:36-44):
        uv = (8 g + 4) / resolution, no jitter."""
        u = div(add(mul(Q(gx), 8), 4), self.res[0])
        v = div(add(mul(Q(gy), 8), 4), self.res[1])
        return self.dir_uv(u, v)

    def dir_uv(self, u, v):
        ndc_x = sub(mul(u, 2), 1)
        ndc_y = sub(1, mul(v, 2))
        aspect = div(self.res[0], self.res[1])
        a = mul(mul(ndc_x, self.tan), aspect)
        b = mul(ndc_y, self.tan)
        r = [add(add(self.forward[k], mul(self.right[k], a)), mul(self.up[k], b))
             for k in range(3)]
        ln = fsqrt(add(add(mul(r[0], r[0]), mul(r[1], r[1])), mul(r[2], r[2])))
        return [div(r[k], ln) for k in range(3)]

    def to_json(self):
        return {"origin": [float(v) for v in self.origin],
                "forward": [float(v) for v in self.forward],
                "right": [float(v) for v in self.right], "up": [float(v) for v in self.up],
                "tan_half_fov": float(self.tan), "res": [int(self.res[0]), int(self.res[1])],
                "jitter": [float(v) for v in self.jitter],
                "world_origin": list(self.world_origin)}


# ---------------------------------------------------------------- geometry


def geometric_first_opaque(sc: Scene, origin, d, t_lo):
    """Exact slab test over the boxes (world coordinates): the smallest entry
    t >= t_lo of a box whose material a first-hit ray stops at, with its
    entry axis and entry voxel.  No traversal state at all."""
    best = None
    for b in sc.boxes:
        m = b[6]
        if m in DECORATION:
            continue
        tn, tf, ax = Q(-10 ** 9), Q(10 ** 9), -1
        ok = True
        for k in range(3):
            lo, hi = Q(b[k]), Q(b[k + 3])
            if d[k] == 0:
                if not (lo <= origin[k] < hi):
                    ok = False
                continue
            a0, a1 = (lo - origin[k]) / d[k], (hi - origin[k]) / d[k]
            if a0 > a1:
                a0, a1 = a1, a0
            if a0 > tn:
                tn, ax = a0, k
            tf = min(tf, a1)
        if not ok or tn >= tf or tf <= t_lo or tn < t_lo:
            continue
        if best is None or tn < best[0]:
            p = [origin[k] + d[k] * tn for k in range(3)]
            vox = [math.floor(p[k]) for k in range(3)]
            vox[ax] = b[ax] if d[ax] > 0 else b[ax + 3] - 1
            best = (tn, ax, vox, m)
    return best


def check_geometry(sc, origin, d, rec, P, exact_t, max_dist=None):
    """Cross-check an emulated first-hit record against exact geometry."""
    max_dist = P.max_dist if max_dist is None else max_dist
    w = Walk(sc, origin, d)
    if not w.valid:
        assert rec["flags"] == 0 and rec["steps"] == 0
        return
    t_in = w.t_enter
    g = geometric_first_opaque(sc, origin, d, t_in)
    tol = (lambda t: Q(0)) if exact_t else (lambda t: Q(1, 10 ** 4) * max(1, abs(t)))
    if rec["flags"] & 1 and rec["t"] == t_in:
        return                          # the walk starts inside a solid voxel
    if rec["flags"] & 1 and not rec["flags"] & 2:
        assert g is not None, (sc.name, rec)
        tn, ax, vox, m = g
        assert rec["mat"] == m and rec["face"] >> 1 == ax, (sc.name, rec, g)
        assert abs(rec["t"] - tn) <= tol(tn), (sc.name, rec, g)
        p = [origin[k] + d[k] * tn for k in range(3)]
        margin = min(abs(p[k] - round(p[k])) for k in range(3) if k != ax)
        if exact_t or margin > Q(1, 1000):
            assert rec["voxel"] == vox, (sc.name, rec, g)
    elif rec["flags"] & 2:
        # an early exit lies no later than the first opaque box along the ray
        if g is not None:
            assert rec["t"] <= g[0] + tol(g[0]), (sc.name, rec, g)
    else:
        # a miss: no opaque box is entered within the distance budget,
        # unless the iteration cap ended the walk
        if g is not None and rec["steps"] < P.max_iters:
            assert g[0] + tol(g[0]) > max_dist, (sc.name, rec, g)


# ---------------------------------------------------------------- the suite

ONE = Q(1)


def dy(num, den_pow):
    return Q(num, 2 ** den_pow)


def worlds():
    # W1: a 1024 x 64 x 256 window (the device world takes whole L4 cells in
    # x and z), ground 8 voxels of stone in z < 64, and per 16-wide z lane a
    # feature along +x.
    lanes = [
        (0, 0, 0, 1024, 8, 64, STONE),                        # ground
        (100, 8, 0, 101, 40, 16, STONE),                      # lane 0: wall at x = 100
        (400, 8, 16, 401, 40, 32, STONE),                     # lane 1: wall at x = 400
        (402, 8, 32, 404, 38, 48, STONE),                     # lane 2: wall at x = 402..403
        (402, 38, 32, 404, 40, 48, DIRT),                     #   with a dirt cap (topmost)
        (512, 16, 48, 516, 20, 52, GRASS),                    # lane 3: one brick low in a tile
        (700, 8, 48, 701, 48, 64, STONE),                     #   and a wall at x = 700
        (520, 8, 0, 521, 40, 16, STONE),                      # lane 0 beyond its first wall
    ]
    w1 = Scene("lanes", (256, 16, 64), (0, 0, 0), lanes)

    # W2: uniform cells, transparency, decoration and far foliage in a
    # 512 x 64 x 256 window at world origin (-300, 0, 1000), so slot x = rel
    # x + 212 (mod 512) and slot z = rel z + 232 (mod 256): a slot tile
    # starts at rel x = 12 and rel z = 8 (mod 16), a slot brick at rel 0
    # (mod 4), and slot z wraps at rel z = 24.
    ro = (-300, 0, 1000)
    X, Z = ro[0], ro[2]

    def rel(x0, y0, z0, x1, y1, z1, m):
        return (X + x0, y0, Z + z0, X + x1, y1, Z + z1, m)
    boxes = [
        rel(0, 0, 0, 512, 4, 64, STONE),            # one brick layer of ground
        rel(76, 16, 8, 92, 32, 24, STONE),          # a uniform slot tile
        rel(64, 16, 16, 68, 20, 20, DIRT),          # a uniform brick before it
        rel(96, 16, 28, 100, 20, 32, GLASS),        # uniform glass (not optimisable)
        rel(104, 16, 28, 108, 20, 32, FLOWER),      # near decoration
        rel(140, 16, 28, 141, 20, 32, DIRT),        # one voxel column behind them
        rel(300, 16, 36, 304, 17, 40, TURF),        # a turf-only brick at t < 400
        rel(440, 16, 36, 444, 17, 40, TURF),        # and one at t > 400 (LOD falls through)
        rel(448, 16, 36, 452, 20, 40, GRASS),       # grass behind it
        rel(300, 40, 36, 304, 44, 40, STONE),       # a stone brick above the first
        rel(200, 24, 48, 202, 26, 50, LEAVES),      # far leaves (t > 128)
        rel(240, 24, 48, 242, 26, 50, WATER),       # near water (t < 400)
        rel(480, 24, 48, 482, 26, 50, WATER),       # far water (t > 400)
        rel(130, 4, 40, 131, 12, 44, GLASS),        # glass then stone, for no-water rays
        rel(132, 4, 40, 133, 12, 44, STONE),
    ]
    w2 = Scene("uniform_shifted", (128, 16, 64), ro, boxes)
    return [w1, w2]


# Hand-derived records.  Each ray runs along +x with a slope of 1/1024 in y
# and 1/2048 in z, so every product and sum of the walk is exact and t is
# the x distance travelled.  Cells are L4 256, chunk 64, tile 16, brick 4.
HAND = [
    # Lane 0, y 20.5, z 8.5, from x 0.5, stock method.
    # it1 (0,20,8): L4 and chunk hold ground; tile x0-15 y16-31 z0-15 empty -> x 16
    # it2 x16, it3 x32, it4 x48: tiles empty (chunk x0-63 holds only ground) -> 64
    # it5 x64 -> 80, it6 x80 -> 96: tiles empty; it7 x96: tile x96-111 holds the
    # wall; brick x96-99 empty -> x 100; it8 (100,20,8): stone.  t = 99.5.
    dict(world="lanes", org=(Q(1, 2), Q(41, 2), Q(17, 2)), d=(ONE, dy(1, 10), dy(1, 11)),
         kind=0, flags=STOCK,
         expect={"voxel": [100, 20, 8], "face": 1, "mat": STONE, "flags": 1, "t": Q(199, 2),
                 "steps": 8}),
    # The same ray with max_dist 99: the iteration at x 100 starts at
    # t_cur 99.5 > 99 and ends the walk; steps 8, a miss.
    dict(world="lanes", org=(Q(1, 2), Q(41, 2), Q(17, 2)), d=(ONE, dy(1, 10), dy(1, 11)),
         kind=0, flags=STOCK, params=dict(max_dist=99),
         expect={"voxel": [0, 0, 0], "face": 255, "mat": 0, "flags": 0, "t": Q(0),
                 "steps": 8}),
    # Lane 1 (z 24.5), y 20.5: tiles x0-383 empty at y16-31 except none ->
    # 24 tile skips reach x 384 (iterations 1-24); it25 x384: tile x384-399
    # empty -> 400; it26 x400: tile holds the wall, brick x400-403 holds it,
    # not uniform, t_cur 399.5 <= 400 so no LOD: voxel (400,20,24) stone.
    dict(world="lanes", org=(Q(1, 2), Q(41, 2), Q(49, 2)), d=(ONE, dy(1, 10), dy(1, 11)),
         kind=0, flags=STOCK,
         expect={"voxel": [400, 20, 24], "face": 1, "mat": STONE, "flags": 1,
                 "t": Q(799, 2), "steps": 26}),
    # Lane 2 (z 40.5), y 37.5 (brick y36-39, dirt cap at y38-39): 25 tile
    # skips reach x 400 (it1-25); it26 x400: brick x400-403 holds the wall at
    # x402; t_cur 399.5 <= 400: voxel (400,37,40) empty -> step (it27 x401,
    # t_cur 400.5 > 400): brick LOD, topmost of the brick = dirt (y 39),
    # recorded at the empty voxel (401,37,40), t 400.5, flags 3.
    dict(world="lanes", org=(Q(1, 2), Q(75, 2), Q(81, 2)), d=(ONE, dy(1, 10), dy(1, 11)),
         kind=0, flags=STOCK,
         expect={"voxel": [401, 37, 40], "face": 1, "mat": DIRT, "flags": 3,
                 "t": Q(801, 2), "steps": 27}),
    # Same ray without LOD: it27 x401 empty, it28 x402 stone (not dirt).
    dict(world="lanes", org=(Q(1, 2), Q(75, 2), Q(81, 2)), d=(ONE, dy(1, 10), dy(1, 11)),
         kind=0, flags=F_L4 | F_LUT,
         expect={"voxel": [402, 37, 40], "face": 1, "mat": STONE, "flags": 1,
                 "t": Q(803, 2), "steps": 28}),
]


def f32_vec(v):
    out = [Q(x) for x in v]
    for x in out:
        assert is_f32(x), v
    return out


def record_json(r):
    return {"voxel": r["voxel"], "face": r["face"], "mat": r["mat"], "flags": r["flags"],
            "t": float(r["t"]), "steps": r["steps"]}


def gen_rays(sc: Scene):
    """The crafted rays of one world: (origin, dir, tmax, kind, params)."""
    out = []
    s10, s11 = dy(1, 10), dy(1, 11)
    if sc.name == "lanes":
        # along +x in each lane at several heights; origins shifted so the
        # hits land just before and after t = 400, 520 and 700
        for lane in range(4):
            z = Q(16 * lane + 8) + Q(1, 2)
            for y in (Q(41, 2), Q(75, 2), Q(57, 2), Q(19, 2) + Q(1, 8)):
                for x0 in (Q(1, 2), Q(-1, 4), Q(9, 4), Q(17, 4), Q(15, 4), Q(-7, 2)):
                    out.append(((x0, y, z), (ONE, s10, s11), None, 0, None))
        # near the distance cut: lane 3 wall at x 700 entered at t 699.75 / 700.25
        for x0 in (Q(1, 4), Q(-1, 4), Q(0) + Q(1, 1024)):
            out.append(((x0, Q(45, 2), Q(113, 2)), (ONE, Q(0), Q(0)), None, 0, None))
            out.append(((x0, Q(45, 2), Q(113, 2)), (ONE, s10, -s11), None, 0,
                        dict(flags=F_L4)))
        # lane 3's low grass brick (x 512) entered from outside the window at
        # t 519.75 (brick LOD) and 520.25 (tile LOD, at the tile's entry)
        for x0 in (Q(-31, 4), Q(-33, 4), Q(-8) + Q(1, 1024)):
            out.append(((x0, Q(35, 2), Q(99, 2)), (ONE, s10, s11), None, 0, None))
            out.append(((x0, Q(35, 2), Q(99, 2)), (ONE, s10, s11), None, 0, dict(flags=F_L4)))
        # -x, diagonal and steep rays, and rays from outside the window
        out.append(((Q(1000) + Q(1, 2), Q(30), Q(24) + Q(1, 4)), (-ONE, -s10, s11), None, 0,
                    None))
        out.append(((Q(3, 2), Q(60) + Q(1, 2), Q(3, 2)), (ONE, -Q(1, 2), Q(1, 4)), None, 0,
                    None))
        out.append(((Q(90) + Q(1, 4), Q(63) + Q(1, 2), Q(7) + Q(1, 2)), (Q(1, 8), -ONE, Q(1, 16)),
                    None, 0, None))
        out.append(((Q(-20) + Q(1, 2), Q(20) + Q(1, 4), Q(8) + Q(1, 2)), (ONE, s10, s11), None, 0,
                    None))
        out.append(((Q(50) + Q(1, 2), Q(100), Q(8) + Q(1, 2)), (Q(1, 4), -ONE, Q(1, 8)), None, 0,
                    None))
        # iteration caps
        for cap in (5, 37):
            out.append(((Q(3, 2), Q(8) + Q(1, 2), Q(3, 2)), (ONE, Q(1, 4), Q(1, 2)), None, 0,
                        dict(max_iters=cap, flags=F_L4)))
        # any-hit and no-water kinds, with their own distance caps
        for tm in (Q(99), Q(100), Q(480), Q(700)):
            out.append(((Q(1, 2), Q(41, 2), Q(17, 2)), (ONE, s10, s11), tm, 1, None))
            out.append(((Q(1, 2), Q(41, 2), Q(17, 2)), (ONE, s10, s11), tm, 2, None))
        out.append(((Q(1, 2), Q(30) + Q(1, 2), Q(60) + Q(1, 2)), (ONE, -Q(1, 64), -s11), Q(480),
                    1, dict(any_max_iters=9)))
    else:
        X, Z = sc.ro[0], sc.ro[2]
        for z in (Q(8) + Q(1, 2), Q(18) + Q(1, 2), Q(29) + Q(1, 2), Q(37) + Q(1, 2),
                  Q(49) + Q(1, 4), Q(42) + Q(1, 2)):
            for y in (Q(18) + Q(1, 2), Q(24) + Q(1, 2), Q(16) + Q(1, 4), Q(25) + Q(1, 8),
                      Q(6) + Q(1, 2), Q(42) + Q(1, 2)):
                for x0 in (Q(1, 2), Q(-5, 4)):
                    o = (Q(X) + x0, y, Q(Z) + z)
                    for kind in (0, 1, 2):
                        tm = None if kind == 0 else Q(700)
                        out.append((o, (ONE, s10, s11), tm, kind, None))
        # -x rays through the wrap of the slot space
        for z in (Q(18) + Q(1, 2), Q(49) + Q(1, 4), Q(37) + Q(1, 2)):
            o = (Q(X + 511) + Q(1, 2), Q(18) + Q(1, 2), Q(Z) + z)
            out.append((o, (-ONE, -s10, s11), None, 0, None))
            out.append((o, (-ONE, -s10, s11), Q(700), 2, None))
        # from above onto the uniform tile, the uniform brick, the glass and
        # the flower
        for (x, z) in ((80, 12), (65, 17), (97, 29), (105, 29)):
            o = (Q(X + x) + Q(1, 4), Q(63) + Q(1, 2), Q(Z + z) + Q(1, 8))
            out.append((o, (Q(1, 32), -ONE, Q(1, 64)), None, 0, None))
            out.append((o, (Q(1, 32), -ONE, Q(1, 64)), Q(700), 2, None))
            out.append((o, (Q(1, 32), -ONE, Q(1, 64)), None, 0, dict(flags=F_L4)))
    return out


def build():
    suite = {"generator": "tests/golden/make_golden.py",
             "record": "voxel (world), face = 2*axis + (step>0) or 255, mat, flags "
                       "(bit0 hit, bit1 early exit), t (binary32), steps (iterations begun)",
             "worlds": [], "rays": [], "frames": [], "picks": []}
    scenes = {sc.name: sc for sc in worlds()}
    for sc in scenes.values():
        suite["worlds"].append(sc.to_json())

    def emit(sc, origin, d, tmax, kind, pov, expect=None, note=None):
        P = Params(**(pov or {}))
        origin = f32_vec(origin)
        d = f32_vec(d)
        tm = P.max_dist if tmax is None else Q(tmax)
        rec = run_kind(sc, origin, d, tm, kind, P)
        exact = all(x.denominator & (x.denominator - 1) == 0 for x in d)
        if kind == 0:
            check_geometry(sc, origin, d, rec, P, exact, tm)
        if expect is not None:
            got = {k: rec[k] for k in expect}
            assert got == expect, (sc.name, origin, d, got, expect)
        pj = P.to_json()
        suite["rays"].append({"world": sc.name, "org": [float(v) for v in origin],
                              "dir": [float(v) for v in d], "tmax": float(tm), "kind": kind,
                              "params": pj, "expect": record_json(rec),
                              "why": note or rec.get("why", "miss")})

    for h in HAND:
        emit(scenes[h["world"]], h["org"], h["d"], None, h["kind"],
             dict(flags=h["flags"], **h.get("params", {})), expect=h["expect"], note="hand")
    skipped = 0
    for sc in scenes.values():
        for (o, d, tm, kind, pov) in gen_rays(sc):
            try:
                emit(sc, o, d, tm, kind, pov)
            except Deviation:
                skipped += 1

    # frames: small cameras looking along +x / down, method without the beam
    # pre-pass and shadow rays (those are checked elsewhere)
    cams = [
        ("lanes", Camera((Q(1, 2), Q(30) + Q(1, 4), Q(32) + Q(1, 8)), (1, 0, 0), (0, 0, 1),
                         (0, 1, 0), Q(3, 64), (16, 9))),
        ("lanes", Camera((Q(380) + Q(1, 2), Q(60), Q(9) + Q(3, 8)),
                         (lit("0.6"), lit("-0.8"), 0), (0, 0, -1), (lit("0.8"), lit("0.6"), 0),
                         Q(1, 2), (12, 8))),
        ("lanes", Camera((Q(-40) + Q(1, 2), Q(21) + Q(1, 2), Q(40) + Q(1, 2)), (1, 0, 0),
                         (0, 0, 1), (0, 1, 0), Q(1, 128), (8, 8), jitter=(Q(1, 4), Q(-1, 8)))),
        ("uniform_shifted", Camera((Q(-300 + 30) + Q(1, 2), Q(40) + Q(1, 4), Q(1000 + 20)),
                                   (1, 0, 0), (0, 0, 1), (0, 1, 0), Q(1, 2), (16, 10),
                                   world_origin=(-300, 0, 1000))),
    ]
    for name, cam in cams:
        sc = scenes[name]
        assert cam.world_origin == sc.ro
        beam = beam_pass(sc, cam)
        for flags in (STOCK, F_L4, STOCK | F_BEAM):
            P = Params(flags=flags)
            recs = []
            W, H = int(cam.res[0]), int(cam.res[1])
            for py in range(H):
                for px in range(W):
                    d = cam.ray_dir(px, py)
                    org, skip = cam.origin, Q(0)
                    if flags & F_BEAM:
                        # cs_main's beam skip (raymarch.wgsl:603-609, :629-631)
                        skip = max(Q(0), sub(beam[py // 8][px // 8], BEAM_MARGIN))
                        org = [add(cam.origin[k], mul(d[k], skip)) for k in range(3)]
                    try:
                        r = trace(sc, org, d, P.max_dist, P)
                    except Deviation:
                        recs.append(None)       # a sub-voxel pixel: not pinned
                        continue
                    if flags & F_BEAM:
                        if r["flags"] & 1:
                            r["t"] = add(r["t"], skip)
                    else:
                        check_geometry(sc, cam.origin, d, r, P, False)
                    recs.append(record_json(r))
            suite["frames"].append({"world": name, "camera": cam.to_json(),
                                    "params": P.to_json(), "expect": recs,
                                    "beam": [[float(b) for b in row] for row in beam]})

    # picking (src/raycast.rs): axis rays and unnormalised oblique ones
    sc = scenes["lanes"]
    picks = [((Q(50) + Q(1, 2), Q(30) + Q(1, 2), Q(8) + Q(1, 2)), (ONE, 0, 0)),
             ((Q(50) + Q(1, 2), Q(30) + Q(1, 2), Q(8) + Q(1, 2)), (Q(3), Q(-4), 0)),
             ((Q(100) + Q(1, 2), Q(20) + Q(1, 2), Q(8) + Q(1, 2)), (ONE, Q(1, 2), 0)),
             ((Q(100) + Q(1, 2), Q(4) + Q(1, 2), Q(8) + Q(1, 2)), (0, ONE, 0)),
             ((Q(10) + Q(1, 2), Q(60) + Q(1, 2), Q(10) + Q(1, 2)), (Q(1, 2), -ONE, Q(1, 4))),
             ((Q(-30), Q(20) + Q(1, 2), Q(8) + Q(1, 2)), (ONE, 0, 0)),
             ((Q(500) + Q(1, 2), Q(70), Q(8) + Q(1, 2)), (0, ONE, 0)),
             ((Q(10) + Q(1, 2), Q(30) + Q(1, 2), Q(70)), (0, 0, -ONE)),
             ((Q(200) + Q(1, 4), Q(50) + Q(3, 4), Q(30) + Q(1, 8)), (Q(-2), Q(-1), Q(1, 2)))]
    for cam, d in picks:
        cam, d = f32_vec(cam), f32_vec(d)
        r = pick(sc, cam, d)
        suite["picks"].append({"world": sc.name, "cam": [float(v) for v in cam],
                               "dir": [float(v) for v in d], "expect": r})
    sc = scenes["uniform_shifted"]
    X, Z = sc.ro[0], sc.ro[2]
    for cam, d in (((Q(X + 60) + Q(1, 2), Q(20) + Q(1, 2), Q(Z + 8) + Q(1, 2)), (ONE, 0, 0)),
                   ((Q(X + 66) + Q(1, 2), Q(18) + Q(1, 2), Q(Z + 18) + Q(1, 2)), (ONE, 0, 0)),
                   ((Q(X + 510) + Q(1, 2), Q(18) + Q(1, 2), Q(Z + 8) + Q(1, 2)), (-ONE, 0, 0)),
                   ((Q(X + 100) + Q(1, 2), Q(30) + Q(1, 2), Q(Z + 18) + Q(1, 2)),
                    (Q(1, 4), -ONE, 0))):
        cam, d = f32_vec(cam), f32_vec(d)
        suite["picks"].append({"world": sc.name, "cam": [float(v) for v in cam],
                               "dir": [float(v) for v in d], "expect": pick(sc, cam, d)})
    suite["skipped_sub_voxel_cases"] = skipped
    return suite


def main():
    suite = build()
    with open(OUT, "w") as f:
        json.dump(suite, f, indent=None, separators=(",", ":"))
        f.write("\n")
    kinds = {}
    for r in suite["rays"]:
        kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
    print(f"{len(suite['rays'])} rays {kinds}, {len(suite['frames'])} frames, "
          f"{len(suite['picks'])} picks, {suite['skipped_sub_voxel_cases']} sub-voxel cases "
          f"left out -> {OUT}")


if __name__ == "__main__":
    sys.exit(main())
