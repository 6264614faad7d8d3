#!/usr/bin/env python
"""Throughput of the voxelG hierarchical-DDA traversal on B200.

Workload (one step = one frame): the 2048x256x2048 seeded world (32x4x32
chunks), 1920x1080 primary rays with the uniform-brick/tile LUTs, the 1/8-res
beam pre-pass and the 400/520-voxel LOD on, plus one shadow ray per primary
hit toward normalize(0.3, 0.8, 0.5) jittered in a 0.5-degree cone.
Every record is bit-exact against the CPU oracle (tests/test_gpu_parity.py).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value      Mrays/s over all ranks (primary + shadow rays), world and rays
           resident in HBM, per-step device time from CUDA events on the
           launching stream, L2 flushed (256 MiB write) before every step
           outside the events, max over ranks.
e2e        the same metric through the host-buffer frame pipeline
           (vx_render_primary_host_async): camera in, every step's records
           copied to pinned host memory inside the timed region, one frame
           rendering while the previous one copies.
roofline   the primary kernel: algorithmic bytes per launch (method loads as
           counted by the oracle's rules + record writes) / mean event time,
           against the measured HBM copy bandwidth.
cpu_baseline  the oracle (C restatement of the reference traversal) on all
           host threads over a bounded row sample of the same frame.

Extra sections (rank 0, single GPU, a few seconds each; --no-extras skips
them), on 512x256x512 worlds:
mixed_queue  primary + spawned shadow + GI-probe + picking rays in one
           autotuned, graph-captured persistent launch.
worldgen   the reference's chunk generator gen_slot_bricks: the criterion
           chunks on one CPU thread beside the device, and whole windows
           (the demo world, a 2048x256x2048 window) on the device.
picking    benches/trace.rs raycast_pick rays on the reference's demo world:
           CPU restatement on one thread (ns/ray) beside batched and
           single-call device picking.
learned    the learned start-distance proposal: on-device training, then the
           plain DDA, the learned form and the verification without a network
           on one 1920x1080 frame, with acceptance and iterations saved.
serving    the ray-query server under 64 open-loop Poisson clients: p50/p99, at the
           north star's load, at a query-sized load where batches form, and past
           capacity with and without continuous batching; then the same three loads
           on the device-resident request loop.
ao         (on the benchmark frame) contact AO of the primary hits.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s bit-exact vs CPU DDA (plain vs learned-proposal); ray-query p50/p99 ms"
UNIT = "Mrays/s"
CONFIG_NAME = "c2"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-seconds", type=float, default=4.0)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-queue, learned and serving workloads")
    ap.add_argument("--profile", action="store_true",
                    help="frames only (one counting pass, warm-up, K timed frames): the "
                         "command profiled with ncu")
    ap.add_argument("--profile-worldgen", action="store_true",
                    help="the chunk generator only (the 512x256x512 demo world once, then K "
                         "fills of the 2048x256x2048 window): the command profiled with ncu")
    ap.add_argument("--profile-queue", action="store_true",
                    help="the mixed ray queue only (512x256x512 world, 4.4M rays, the "
                         "tuning 256 threads / refill at 32 idle lanes / coherence sort, K "
                         "graph launches): the command profiled with ncu")
    ap.add_argument("--profile-learned", action="store_true",
                    help="the learned-form frames only (a short training, then K plain, "
                         "learned and verification-only frames): the command profiled "
                         "with ncu")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        gpu_index = ids[local_index] if local_index < len(ids) else str(local_index)
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200", "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 10:
                continue
            m = re.match(r"\s*(\d+)", r[2])
            if m:
                sm.append(int(m.group(1)))
            m = re.match(r"\s*(\d+)", r[3])
            if m:
                smax.append(int(m.group(1)))
            for name, v in zip(names, r[6:10]):
                if "Active" in v and "Not" not in v:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    """HBM copy bandwidth of this pool's B200s: MEASURED_PEAKS.json's hbm_gbs
    (a number, or an object holding one) when the file is there and readable,
    else the earlier measurement of 6.65 TB/s."""
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        v = json.loads(p.read_text()).get("hbm_gbs")
        if isinstance(v, dict):
            v = next((v[k] for k in ("value", "burst", "gbs", "measured") if k in v), None)
        if isinstance(v, (int, float)) and v > 0:
            return {"hbm_gbs": float(v), "source": "measured"}
    except (OSError, ValueError, AttributeError):
        pass
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled(key: str) -> float | None:
    """A per-launch figure of the primary kernel from the committed ncu
    summary (profiles/primary_c2_1080p.md): `traffic_bytes_per_launch` (dram
    bytes read + written) or `warp_instructions_per_launch`
    (smsp__inst_executed.sum), if present."""
    p = ROOT / "profiles" / "primary_c2_1080p.md"
    if not p.exists():
        return None
    m = re.search(key + r":\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


def dist_setup(n_gpus: int):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(world: int, rays_per_step: int, steps: int, dev_ms: float, device):
    """Whole-job throughput in Mrays/s: every rank renders rays_per_step per
    step (weak scaling) and the job takes as long as the slowest rank's
    device time.  Returns (max device ms over ranks, value)."""
    dev_ms_max = max_over_ranks(dev_ms, world, device)
    return dev_ms_max, world * rays_per_step * steps / (dev_ms_max / 1e3) / 1e6


def frame_setup(vg, cfg, device: int):
    dw = vg.DeviceWorld(*cfg.bricks, device=device)
    dw.generate(cfg.terrain)
    cam = vg.default_camera(dw, cfg.width, cfg.height)
    params = vg.default_params(cfg.flags, frame=7.0)
    return dw, cam, params


# -------------------------------------------------------------- cpu sample
def cpu_sample(ow, cam, params, seconds: float, threads: int):
    """Time the oracle on whole frames (beam pre-pass, every primary ray and
    its shadow ray; rows handed out to the threads one at a time), repeated
    until about `seconds` of wall time.  Returns (Mrays/s, frames, seconds)."""
    from oracle import pyoracle as po
    total_rays, total_s, frames = 0, 0.0, 0
    while True:
        rec, sh, _, secs, _ = po.render_frame(ow, cam, params, threads=threads)
        total_rays += len(rec) + int(sh["traced"].sum())
        total_s += secs
        frames += 1
        if total_s >= seconds:
            break
    return total_rays / total_s / 1e6, frames, total_s


def run_reference(args, cfg):
    """The reference's CPU traversal (the oracle restatement: the Rust
    reference cannot be built here) on all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import math

    from oracle import pyoracle as po
    threads = os.cpu_count() or 1
    ow = po.World(*cfg.bricks)
    ow.generate(cfg.terrain, threads=threads)
    # camera + params built on the oracle side: nothing of libvoxrt runs here
    cx, cz = cfg.bricks[0] * 2, cfg.bricks[2] * 2
    cam = po.camera_from_pose((cx, 140.0, cz), 0.0, math.radians(-15.0), math.radians(70.0),
                              cfg.width, cfg.height)
    params = po.default_params(cfg.flags, frame=7.0)
    # one step = the whole frame, as the device arm renders it: beam
    # pre-pass, every primary ray and its shadow ray, rows handed out to all
    # host threads one at a time
    per_step = []
    rays_step = []
    for s in range(args.warmup + args.steps):
        rec, sh, _, secs, _ = po.render_frame(ow, cam, params, threads=threads)
        if s >= args.warmup:
            per_step.append(secs)
            rays_step.append(len(rec) + int(sh["traced"].sum()))
    value = sum(rays_step) / sum(per_step) / 1e6
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.mean(per_step), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{CONFIG_NAME}: 2048x256x2048 world, 1920x1080 primary + shadow "
                               "rays, beam/LUT/LOD on", "sample": "the whole frame every step"},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads,
                         "kind": "port",
                         "sample": f"the whole 1920x1080 frame per step (beam pre-pass, "
                                   f"{int(sum(rays_step) / len(rays_step))} primary + shadow "
                                   "rays), C restatement of the reference traversal (the Rust "
                                   "reference cannot be built here)"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------- extras
def run_picking(vg, dw, n: int = 200_000) -> dict:
    """The reference's criterion picking case (benches/trace.rs:24-40: origin
    (256, 90, 256), dir (sin a, -0.5, cos a), a += 0.013) on the world it
    picks in, World::new + fill_demo_terrain (seed 0xC0FFEE_F00D_BEEF,
    512x256x512): the CPU baseline (the raycast restatement, one thread,
    as criterion runs it) beside the device -- batched rays (event time) and
    the single-ray drop-in call (wall time per call, copies and sync
    included)."""
    import ctypes as C

    import numpy as np
    import torch

    from oracle import pyoracle as po
    from voxelg_b200 import _lib as L

    a = (np.arange(1, n + 1, dtype=np.float32) * np.float32(0.013)).astype(np.float32)
    dirs = np.stack([np.sin(a), np.full(n, -0.5, np.float32), np.cos(a)], 1).astype(np.float32)
    cams = np.tile(np.array([256.0, 90.0, 256.0], np.float32), (n, 1))
    ow = po.World(*dw.dims, arrays=dw.download())
    want, whit, cpu_s = po.raycast_batch(ow, cams, dirs, threads=1)
    del ow
    dev = torch.device("cuda", dw.device)
    c = torch.from_numpy(cams.reshape(-1)).to(dev)
    d = torch.from_numpy(dirs.reshape(-1)).to(dev)
    out = torch.empty(n * 24, dtype=torch.uint8, device=dev)
    hit = torch.empty(n, dtype=torch.int32, device=dev)
    lib = L.load()
    stream = torch.cuda.current_stream(dev).cuda_stream

    def batch():
        L.check(lib.vx_raycast_batch(dw.handle, L.i3((0, 0, 0)), C.c_void_p(c.data_ptr()),
                                     C.c_void_p(d.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                     C.c_void_p(hit.data_ptr()), C.c_void_p(stream)))
    for _ in range(3):
        batch()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        batch()
    e1.record()
    torch.cuda.synchronize(dev)
    gpu_ns = e0.elapsed_time(e1) / 10 * 1e6 / n
    same = bool(np.array_equal(out.cpu().numpy(), want.view(np.uint8).reshape(-1)) and
                np.array_equal(hit.cpu().numpy(), whit))
    pick = L.VxPickHit()
    calls = 2000
    for i in range(20):
        lib.vx_raycast(dw.handle, L.f3(cams[i]), L.f3(dirs[i]), L.i3((0, 0, 0)), C.byref(pick))
    t0 = time.perf_counter()
    for i in range(calls):
        lib.vx_raycast(dw.handle, L.f3(cams[i]), L.f3(dirs[i]), L.i3((0, 0, 0)), C.byref(pick))
    single_us = (time.perf_counter() - t0) / calls * 1e6
    return {
        "workload": f"benches/trace.rs raycast_pick rays x {n} on the reference's demo world "
                    "(fill_demo_terrain, seed 0xC0FFEE_F00D_BEEF, 512x256x512)",
        "cpu_1thread_ns_per_ray": round(cpu_s * 1e9 / n, 1),
        "gpu_batch_ns_per_ray": round(gpu_ns, 3),
        "gpu_single_call_us": round(single_us, 2),
        "hits": int(whit.sum()), "equal_to_cpu": same,
    }


def run_learned(vg, dw) -> dict:
    """Learned start-distance proposal on the 512x256x512 world at 1920x1080:
    train on the device (16.4M plain-DDA pairs from 200 poses), then time the
    plain DDA, the learned form and the verification without a network on
    the same frame (primary rays, method flags L4|LUT|LOD, no beam), and
    check that all three give the same records except steps.  Each form is
    timed over `reps` frames enqueued back to back between two CUDA events
    on the launching stream (no statistics collected in the timed frames);
    a separate call collects the form's statistics."""
    import numpy as np
    import torch

    from voxelg_b200 import _lib as L
    from voxelg_b200 import learned as vl

    cam = vg.default_camera(dw, 1920, 1080)
    p = vg.default_params(L.VX_F_L4 | L.VX_F_LUT | L.VX_F_LOD)
    n = 1920 * 1080
    st = torch.cuda.current_stream()
    stream = st.cuda_stream
    prop = vl.Proposal(dw, seed=7)
    cfg = vl.default_config()
    t0 = time.perf_counter()
    curve, held_before, held_after = prop.train(dw, cfg)
    train_s = time.perf_counter() - t0
    plain = torch.empty(n * 24, dtype=torch.uint8, device="cuda")
    rec = torch.empty_like(plain)
    reps = 20

    def batch_ms(frame):
        """Mean ms per frame of `reps` frames enqueued back to back."""
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

    plain_ms = min(batch_ms(lambda: vg.render_primary(dw, cam, p, plain, stream=stream))
                   for _ in range(3))
    torch.cuda.synchronize()
    a = vg.records(plain)
    plain_iters = int(a["steps"].astype(np.int64).sum())
    res = {}
    for name, pr in (("learned", prop), ("verify_only", None)):
        ms = min(batch_ms(lambda: vl.render_learned(dw, pr, cam, p, rec, stats=False,
                                                    stream=stream)) for _ in range(3))
        s = vl.render_learned(dw, pr, cam, p, rec, stream=stream)
        b = vg.records(rec)
        fa, fb = a.copy(), b.copy()
        fa["steps"] = 0
        fb["steps"] = 0
        res[name] = {
            "ms": round(ms, 4), "infer_ms_in_stats_call": round(s.infer_ms, 4),
            "mrays_s": round(n / ms / 1e3, 1), "speedup_vs_plain": round(plain_ms / ms, 3),
            "iters_per_ray": round(s.iters / n, 3),
            "steps_saved_per_ray": round((plain_iters - s.iters) / n, 3),
            "ray_checks_per_ray": round(s.cells / n, 3),
            "acceptance": round(s.accepted / n, 4), "partial": round(s.partial / n, 4),
            "verified_miss": round(s.miss / n, 4), "unverified": round(s.none / n, 4),
            "fallback": int(s.fallback),
            "records_equal_except_steps": bool(np.array_equal(fa.view(np.uint8),
                                                              fb.view(np.uint8))),
        }
    prop.close()
    return {
        "workload": "512x256x512 world, 1920x1080 primary rays, method L4|LUT|LOD without the "
                    "beam; MLP 70-64-64-64-1 GELU trained on 16.4M plain-DDA pairs (200 poses); "
                    "one proposal and one frustum proof per 8x4 pixel tile",
        "timing": f"mean of {reps} frames enqueued back to back between CUDA events, best of 3",
        "train_s": round(train_s, 3), "train_steps": int(cfg.steps),
        "held_out_loss_before": round(held_before, 4), "held_out_loss_after": round(held_after, 4),
        "plain_ms": round(plain_ms, 4), "plain_mrays_s": round(n / plain_ms / 1e3, 1),
        "plain_iters_per_ray": round(plain_iters / n, 3), **res,
    }


def run_worldgen(vg, device: int) -> tuple:
    """The reference's chunk generator gen_slot_bricks (src/voxel.rs:1322-1500).
    The criterion case (benches/trace.rs:11-22: chunks (i & 7, 0, (i >> 3) & 7),
    seed 0xC0FFEE_F00D_BEEF) runs on one CPU thread through the oracle
    restatement, as criterion runs it, and on the device as one batch;
    whole windows are the 512x256x512 demo world (fill_demo_terrain, 2048
    chunks) and a 2048x256x2048 window (32768 chunks).  Device figures are
    wall times of the synchronous call: job upload, generation and pyramid
    rebuild.  Returns (result, the demo world for the picking case)."""
    import numpy as np

    from oracle import pyoracle as po

    seed = 0xC0FFEE_F00D_BEEF
    chunks = [(i & 7, 0, (i >> 3) & 7) for i in range(1, 65)]
    t0 = time.perf_counter()
    want = [po.gen_slot_bricks(*c, seed) for c in chunks for _ in range(2)][::2]
    cpu_ns = (time.perf_counter() - t0) / (2 * len(chunks)) * 1e9
    demo = vg.DeviceWorld(128, 64, 128, device=device)

    def wall(fn, reps):
        fn()
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t) / reps

    # the criterion chunks: slots (x, 0, z) of the demo window, x, z < 8
    batch_s = wall(lambda: demo.gen_chunks(seed, chunks), 10)
    got = demo.download()["bricks"].reshape(128, 64, 128)   # (z, y, x) bricks
    same = all(np.array_equal(
        np.ascontiguousarray(got[cz * 8:cz * 8 + 8, 0:8, cx * 8:cx * 8 + 8]).reshape(-1)
        .view(np.uint8), w.reshape(-1).view(np.uint8)) for (cx, _, cz), w in zip(chunks, want))
    demo_s = wall(lambda: demo.fill_window(seed, 0, 0), 5)
    big = vg.DeviceWorld(512, 64, 512, device=device)
    big_s = wall(lambda: big.fill_window(seed, 0, 0), 3)
    big.close()
    return {
        "workload": "gen_slot_bricks (terrain, biomes, ores, decoration, trees), seed "
                    "0xC0FFEE_F00D_BEEF",
        "criterion_case": {"chunks": len(chunks), "cpu_1thread_us_per_chunk":
                           round(cpu_ns / 1e3, 1), "gpu_us_per_chunk":
                           round(batch_s * 1e6 / len(chunks), 2), "equal_to_cpu": same},
        "demo_world_512x256x512": {"chunks": 2048, "ms": round(demo_s * 1e3, 3),
                                   "chunks_per_s": round(2048 / demo_s)},
        "window_2048x256x2048": {"chunks": 32768, "ms": round(big_s * 1e3, 3),
                                 "chunks_per_s": round(32768 / big_s)},
    }, demo


def run_extras(vg, device: int) -> dict:
    """The other workloads on the 512x256x512 world, each a few seconds:
    the mixed ray queue (one autotuned, graph-captured persistent launch),
    the criterion picking case, the learned proposal and the ray-query
    serving loop (64 Poisson clients)."""
    import torch

    import voxelg_b200.queue as q
    import voxelg_b200.serve as sv
    from voxelg_b200 import _lib as L

    out = {}
    c1 = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*c1.bricks, device=device)
    dw.generate(c1.terrain)
    cam = vg.default_camera(dw, 1920, 1080)
    rays, counts = q.mixed_queue(c1.bricks, cam, 1920, 1080, seed=11)
    p = vg.default_params(L.VX_F_L4 | L.VX_F_LUT | L.VX_F_LOD, frame=7.0)
    best, tune_ms, rt, o, sh = q.autotune(dw, rays, p, reps=3)
    g = q.Graph(dw, rt, p, tuning=best)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        g.launch(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record()
    for _ in range(reps):
        g.launch(stream)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    n_sh = int(vg.shadows(g.shadow)["traced"].sum())
    out["mixed_queue"] = {
        "workload": "512x256x512 world: 1920x1080 primary rays + their shadow rays, GI probes "
                    "on a 16-voxel grid within 256 voxels (64 Fibonacci rays, max 256), "
                    "10k picking rays (max 8), seeded shuffle; one graph-captured launch",
        "rays": len(rays) + n_sh, "queue_rays": len(rays), "spawned_shadow_rays": n_sh,
        "counts": counts, "ms_per_launch": round(ms, 4),
        "mrays_s": round((len(rays) + n_sh) / ms / 1e3, 2),
        "tuning": {"block_threads": best.block_threads, "refill_min": best.refill_min,
                   "sort": best.sort}, "autotune_best_ms": round(tune_ms, 4),
    }
    g.close()
    del rt, o, sh
    out["worldgen"], demo = run_worldgen(vg, device)
    out["picking"] = run_picking(vg, demo)
    demo.close()
    out["learned"] = run_learned(vg, dw)
    def serve(rate, max_rays, max_len, max_req=0, resident=False):
        srv = sv.Server(dw, p, mem_budget_bytes=1 << 30, slots=8, max_batch_requests=max_req,
                        resident=resident)
        st = srv.bench(clients=64, rate_per_client=rate, seconds=3.0, min_rays=1,
                       max_rays=max_rays, min_len=8.0, max_len=max_len,
                       edit_fraction_per_s=0.01, seed=3)
        srv.close()
        r = {"requests": st["requests"], "p50_ms": round(st["p50_ms"], 4),
             "p99_ms": round(st["p99_ms"], 4), "max_ms": round(st["max_ms"], 4),
             "mrays_s": round(st["mrays_per_s"], 2), "edits": st["edits"],
             "seconds": round(st["seconds"], 2)}
        if resident:
            # launches of the loop: one per edit (an edit ends the launch), per
            # idle gap and per quarter second
            r["loop_launches"] = st["batches"]
        else:
            r["batches"] = st["batches"]
            r["requests_per_batch"] = round(st["requests"] / max(1, st["batches"]), 2)
        return r

    # the north star's load: large requests, the offered load well below capacity
    out["serving"] = {
        "workload": "64 clients, Poisson 200 req/s each, 1-50k rays per request (log-uniform), "
                    "max length 8-512, 1% of bricks re-randomized per second",
        **serve(200.0, 50000, 512.0)}
    # query-sized requests (picking, line of sight) at a rate where batches form
    out["serving_batched"] = {
        "workload": "64 clients, Poisson 2000 req/s each, 1-4000 rays per request "
                    "(log-uniform), max length 8-256, 1% of bricks re-randomized per second",
        **serve(2000.0, 4000, 256.0)}
    # the same requests past saturation: continuous batching against one request
    # per batch (max_batch_requests = 1), the server's capacity either way
    sat = serve(4000.0, 4000, 256.0)
    one = serve(4000.0, 4000, 256.0, max_req=1)
    out["serving_saturated"] = {
        "workload": "64 clients, Poisson 4000 req/s each (past capacity: each client keeps 4 "
                    "requests in flight), 1-4000 rays per request, max length 8-256",
        "batched": sat, "one_request_per_batch": one,
        "batching_gain": round(sat["mrays_s"] / max(1e-9, one["mrays_s"]), 3)}
    # the device-resident request loop (VX_SERVE_RESIDENT) under the same three loads
    out["serving_resident"] = {
        "workload": "the loads of serving, serving_batched and serving_saturated, served by "
                    "the device-resident request loop (one persistent launch takes requests "
                    "from mapped host memory; page-locked client buffers read and written "
                    "in place)",
        "north_star_load": serve(200.0, 50000, 512.0, resident=True),
        "query_load": serve(2000.0, 4000, 256.0, resident=True),
        "past_capacity": serve(4000.0, 4000, 256.0, resident=True)}
    dw.close()
    return out


# ----------------------------------------------------------------- ours
def run_ours(args, cfg):
    import numpy as np
    import torch

    import voxelg_b200 as vg
    from voxelg_b200 import _lib as L

    rank, world, local = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    dw, cam, params = frame_setup(vg, cfg, local)
    W, H = cfg.width, cfg.height
    n = W * H
    rec = torch.empty(n * 24, dtype=torch.uint8, device=device)
    sh = torch.empty(n * 8, dtype=torch.uint8, device=device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream

    # algorithmic bytes of one frame (counting pass, untimed)
    stats = vg.render_stats(dw, cam, params)
    vg.render_primary(dw, cam, params, rec, sh, stream=stream)
    torch.cuda.synchronize(device)
    shadows = vg.shadows(sh)
    n_shadow = int(shadows["traced"].sum())
    rays_per_step = n + n_shadow
    record_bytes = n * (24 + 8)

    for _ in range(max(args.warmup, 3)):
        vg.render_primary_timed(dw, cam, params, rec, sh, stream=stream)

    if args.profile:
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            ms.append(sum(vg.render_primary_timed(dw, cam, params, rec, sh, stream=stream)))
        print(json.dumps({"profile_frames": args.steps, "ms_per_frame": statistics.mean(ms),
                          "rays_per_frame": rays_per_step}), flush=True)
        dw.close()
        return

    sampler = ClockSampler(local) if rank == 0 or world > 1 else None
    barrier(world)
    torch.cuda.synchronize(device)
    beam_ms, prim_ms = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        b, p = vg.render_primary_timed(dw, cam, params, rec, sh, stream=stream)
        beam_ms.append(b)
        prim_ms.append(p)
    torch.cuda.synchronize(device)
    barrier(world)
    wall = time.perf_counter() - t0
    clocks = sampler.stop() if sampler else None
    dev_ms = sum(beam_ms) + sum(prim_ms)
    dev_ms_max, value = aggregate(world, rays_per_step, args.steps, dev_ms, device)

    # end to end through the host-buffer entry points: a frame pipeline, each
    # step's results copied into one of two pinned host buffers while the
    # next frame renders, every copy inside the timed region.  The headline
    # delivers compact records (vx_render_primary_host_compact_async: 12
    # bytes per pixel holding the record and the shadow record without loss);
    # the same pipeline with 16-byte packed records and with the full 24 +
    # 8-byte records is timed beside it.
    cp_h = [torch.empty(n * 12, dtype=torch.uint8).pin_memory() for _ in range(2)]
    cp_np = [r.numpy().view(L.COMPACT_DTYPE) for r in cp_h]
    pk_h = [torch.empty(n * 16, dtype=torch.uint8).pin_memory() for _ in range(2)]
    pk_np = [r.numpy().view(L.PACKED_DTYPE) for r in pk_h]
    rec_h = [torch.empty(n * 24, dtype=torch.uint8).pin_memory() for _ in range(2)]
    sh_h = [torch.empty(n * 8, dtype=torch.uint8).pin_memory() for _ in range(2)]
    rec_np = [r.numpy().view(L.RECORD_DTYPE) for r in rec_h]
    sh_np = [r.numpy().view(L.SHADOW_DTYPE) for r in sh_h]
    e2e_steps = max(40, min(args.steps, 200))   # PCIe-bound: a longer sample steadies it

    def pipeline(enqueue, steps):
        for i in range(3):
            enqueue(i)
        vg.render_host_wait(dw)
        barrier(world)
        torch.cuda.synchronize(device)
        t = time.perf_counter()
        for i in range(steps):
            enqueue(i)
        vg.render_host_wait(dw)
        torch.cuda.synchronize(device)
        barrier(world)
        return max_over_ranks(time.perf_counter() - t, world, device)

    e2e_s = pipeline(lambda i: vg.render_primary_host_compact_async(dw, cam, params,
                                                                    cp_np[i & 1]), e2e_steps)
    e2e_value = world * rays_per_step * e2e_steps / e2e_s / 1e6
    pk_s = pipeline(lambda i: vg.render_primary_host_packed_async(dw, cam, params, pk_np[i & 1]),
                    e2e_steps)
    e2e_packed_value = world * rays_per_step * e2e_steps / pk_s / 1e6
    full_s = pipeline(lambda i: vg.render_primary_host_async(dw, cam, params, rec_np[i & 1],
                                                             sh_np[i & 1]), e2e_steps)
    e2e_full_value = world * rays_per_step * e2e_steps / full_s / 1e6
    want = rec.cpu().numpy()
    want_sh = sh.cpu().numpy()
    assert all(np.array_equal(r.numpy(), want) for r in rec_h), "host path differs from device"
    window = tuple(4 * b for b in cfg.bricks)
    for pk in pk_np:
        r2, s2 = vg.unpack_records(pk, tuple(cam.world_origin), window)
        assert r2.tobytes() == want.tobytes() and s2.tobytes() == want_sh.tobytes(), \
            "packed host records differ from the device records"
    for cp in cp_np:
        r2, s2 = vg.unpack_compact_records(cp, tuple(cam.world_origin), window)
        assert r2.tobytes() == want.tobytes() and s2.tobytes() == want_sh.tobytes(), \
            "compact host records differ from the device records"
    t_up = time.perf_counter()
    vg.unpack_compact_records(cp_np[0], tuple(cam.world_origin), window)
    unpack_ms = (time.perf_counter() - t_up) * 1e3
    # the synchronous calls, for reference
    t2 = time.perf_counter()
    for _ in range(10):
        vg.render_primary_host_compact(dw, cam, params, cp_np[0])
    e2e_sync_value = rays_per_step * 10 / (time.perf_counter() - t2) / 1e6

    peaks = measured_peaks()
    prim_mean = statistics.mean(prim_ms)
    alg_bytes = stats["primary"][0] + record_bytes
    achieved = alg_bytes / (prim_mean / 1e3) / 1e9
    traffic = profiled("traffic_bytes_per_launch")
    # issue roofline: k_primary's warp instructions per launch (ncu) over the
    # issue slots of its event-timed duration -- 4 schedulers per SM, one
    # warp instruction per scheduler per cycle, at the SM clock sampled in
    # the timed region
    warp_inst = profiled("warp_instructions_per_launch")
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    issue_peak = sms * 4 * sm_mhz * 1e6
    issue_achieved = warp_inst / (prim_mean / 1e3) if warp_inst else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import pyoracle as po
        arrays = dw.download()
        ow = po.World(*cfg.bricks, arrays=arrays)
        threads = os.cpu_count() or 1
        cval, frames, secs = cpu_sample(ow, cam, params, args.cpu_sample_seconds, threads)
        cpu = {"value": round(cval, 3), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{frames} whole frames of the same workload (beam pre-pass, primary "
                         f"and shadow rays), {secs:.1f} s wall on {threads} threads; C "
                         "restatement of the reference traversal (the Rust reference cannot "
                         "be built here)"}
        del ow, arrays

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        # contact AO of the benchmark frame's primary hits (12 neighbour tests
        # per hit within 64 voxels), timed alone on the frame's records
        ao = torch.empty(n, dtype=torch.float32, device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            vg.render_ao(dw, cam, rec, ao, stream=stream)
        e0.record()
        for _ in range(20):
            vg.render_ao(dw, cam, rec, ao, stream=stream)
        e1.record()
        torch.cuda.synchronize(device)
        ao_ms = e0.elapsed_time(e1) / 20
        extras["ao"] = {"workload": "contact AO of the 1920x1080 frame's primary hits "
                                    "(vx_render_ao on the frame's records)",
                        "ms": round(ao_ms, 4), "mpixels_s": round(n / ao_ms / 1e3, 1),
                        "occluded_fraction": round(float((ao < 1.0).float().mean()), 4)}
        extras.update(run_extras(vg, local))

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dev_ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": f"{CONFIG_NAME}: 2048x256x2048 world (32x4x32 chunks, seed "
                            f"{cfg.terrain.seed:#x}), 1920x1080 primary rays, beam/LUT/LOD on, "
                            "one shadow ray per hit",
                "rays_per_step": rays_per_step, "primary_rays": n, "shadow_rays": n_shadow,
                "primary_mrays_s": round(world * n * args.steps / (dev_ms_max / 1e3) / 1e6, 3),
                "beam_ms": round(statistics.mean(beam_ms), 4),
                "primary_ms": round(prim_mean, 4),
                "wall_s_timed_loop": round(wall, 3),
                "l2": "flushed before every step (256 MiB write, outside the step events)",
                "parallelism": f"replicas: {world} x full frame (weak scaling)",
            },
            "roofline": {
                "bound": "issue",
                "achieved": round(issue_achieved / 1e9, 2) if issue_achieved else None,
                "peak": round(issue_peak / 1e9, 2), "unit": "G warp-inst/s",
                "frac": round(issue_achieved / issue_peak, 4) if issue_achieved else None,
                "traffic": traffic, "kernel": "k_primary (trace + shadow)",
                "warp_instructions_per_launch": warp_inst,
                "issue_peak_basis": f"{sms} SMs x 4 schedulers x {sm_mhz:.0f} MHz (median "
                                    "sampled in the timed region)",
                "effective_gbs": round(achieved, 2), "hbm_peak_gbs": peaks["hbm_gbs"],
                "hbm_frac": round(achieved / peaks["hbm_gbs"], 4),
                "algorithmic_bytes_per_launch": alg_bytes,
                "peak_source": peaks["source"],
                "note": "bytes the method reads by the reference's widths (1.4 GB) come "
                        "from L1/L2; DRAM traffic per launch is `traffic`; the kernel is "
                        "bound by instruction issue (integer ALU pipe), not HBM"},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                    "h2d_bytes_per_step": 80 + 76,
                    "d2h_bytes_per_step": 12 * n,
                    "api": "vx_render_primary_host_compact_async: frame pipeline, two pinned "
                           "host buffers, every step's compact records (12 B per pixel: "
                           "record and shadow record, lossless) copied in the timed region",
                    "synchronous_call_value": round(e2e_sync_value, 3),
                    "packed_records_value": round(e2e_packed_value, 3),
                    "packed_records_api": "vx_render_primary_host_packed_async (16 B per pixel)",
                    "full_records_value": round(e2e_full_value, 3),
                    "full_records_d2h_bytes_per_step": record_bytes,
                    "full_records_api": "vx_render_primary_host_async (24 + 8 B per pixel)",
                    "host_unpack_ms": round(unpack_ms, 3),
                    "packed_equals_full": True, "compact_equals_full": True},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
        if cpu:
            out["cpu_baseline"] = cpu
        out.update(extras)
        print(json.dumps(out), flush=True)
    dw.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def profile_learned(args):
    """K frames of each form on the 512x256x512 world at 1920x1080 after a
    short training (20 poses, 200 steps): the launches ncu captures."""
    import torch

    import voxelg_b200 as vg
    from voxelg_b200 import learned as vl
    c1 = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*c1.bricks)
    dw.generate(c1.terrain)
    cam = vg.default_camera(dw, 1920, 1080)
    p = vg.default_params(7)
    prop = vl.Proposal(dw, seed=7)
    prop.train(dw, vl.default_config(poses=20, rays_per_pose=16384, steps=200,
                                     held_out_poses=0))
    rec = torch.empty(1920 * 1080 * 24, dtype=torch.uint8, device="cuda")
    for _ in range(args.steps):
        vg.render_primary(dw, cam, p, rec)
        vl.render_learned(dw, prop, cam, p, rec, stats=False)
        vl.render_learned(dw, None, cam, p, rec, stats=False)
    torch.cuda.synchronize()
    print(json.dumps({"profile_learned_frames": args.steps}), flush=True)
    prop.close()
    dw.close()


def profile_queue(args):
    """The mixed ray queue's launches for ncu: the workload of the
    mixed_queue section, captured once in a graph and launched K times."""
    import torch

    import voxelg_b200 as vg
    import voxelg_b200.queue as q
    from voxelg_b200 import _lib as L
    c1 = vg.CONFIGS["c1"]
    dw = vg.DeviceWorld(*c1.bricks)
    dw.generate(c1.terrain)
    cam = vg.default_camera(dw, 1920, 1080)
    rays, _ = q.mixed_queue(c1.bricks, cam, 1920, 1080, seed=11)
    p = vg.default_params(L.VX_F_L4 | L.VX_F_LUT | L.VX_F_LOD, frame=7.0)
    t = q.default_tuning()
    t.block_threads, t.refill_min, t.ctas_per_sm, t.sort = 256, 32, 0, 1
    g = q.Graph(dw, rays, p, tuning=t)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(args.steps):
        g.launch(stream)
    torch.cuda.synchronize()
    print(json.dumps({"profile_queue_launches": args.steps}), flush=True)
    g.close()
    dw.close()


def profile_worldgen(args):
    """The chunk generator's launches for ncu: the 512x256x512 demo world
    (2048 chunks) once, then K fills of the 2048x256x2048 window (32768
    chunks), seed 0xC0FFEE_F00D_BEEF."""
    import voxelg_b200 as vg
    seed = 0xC0FFEE_F00D_BEEF
    demo = vg.DeviceWorld(128, 64, 128)
    demo.fill_window(seed, 0, 0)
    demo.close()
    big = vg.DeviceWorld(512, 64, 512)
    for _ in range(args.steps):
        big.fill_window(seed, 0, 0)
    big.close()
    print(json.dumps({"profile_worldgen_fills": args.steps}), flush=True)


def main():
    args = parse_args()
    import voxelg_b200.configs as configs
    cfg = configs.CONFIGS[CONFIG_NAME]
    if args.profile_learned:
        profile_learned(args)
        return
    if args.profile_worldgen:
        profile_worldgen(args)
        return
    if args.profile_queue:
        profile_queue(args)
        return
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
