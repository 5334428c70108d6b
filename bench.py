#!/usr/bin/env python
"""Benchmark of the RKIField SDF ray-march hot path on B200.

Workload: the large seeded scene (512 primitives in a 256 m cube, voxelized
at 2 cm into ~500k 8^3 f16 bricks, two-level brick index) and one
1920x1080 primary view per step.  ``value`` is Mrays/s of the B200 march
(``rkf_march``) with the scene and outputs resident in HBM, timed with CUDA
events on the launching stream; L2 is flushed (256 MiB write) between steps
outside the timed events.  ``e2e`` is the same metric through the public
host-buffer call (G-buffer copied back to pinned host memory every step).
``plain`` is the one-launch-per-request reference-layout kernel on the same
rays; ``cpu_baseline`` the CPU restatement of the shader on the host cores.

Multi-GPU: the march does not exchange data between rays, so N>1 runs N
independent replicas (one per GPU), each marching its own view of the same
scene; value = all rays / max over ranks of the device time.

``--impl reference`` times the reference algorithm's CPU implementation
(the restatement of ray_march.wgsl; the WGSL pass itself cannot run
without a graphics stack) on all host threads, on a bounded ray sample.
"""
from __future__ import annotations

import argparse
import contextlib
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from rkifield_b200 import _abi as abi  # noqa: E402
from rkifield_b200 import scenes  # noqa: E402

METRIC = "Mrays/s + p99 latency: served/batched vs plain march, 1 B200, Δt≤0.01 voxel"
LARGE_POOL = 3_000_000  # brick slots reserved for the large scene (~20 GB with the reference AoS copy)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scene", default="large", choices=["large", "small"])
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--cpu-rows", type=int, default=24, help="rows of the view in the CPU sample")
    ap.add_argument("--sector-rows", type=int, default=16, help="rows used to count algorithmic sectors")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-sectors", action="store_true")
    ap.add_argument("--extras", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the 960x540 view and the f32 / u8 planes")
    ap.add_argument("--cb-views", type=int, default=64, help="views in the batching workload (0 = skip)")
    ap.add_argument("--cb-steps", type=int, default=3)
    ap.add_argument("--cs-requests", type=int, default=600, help="requests in the serving run (0 = skip)")
    ap.add_argument("--cs-rate", type=float, default=2000.0, help="the serving workload's offered rate")
    ap.add_argument("--cs-rates", default="5000,10000,20000",
                    help="further offered rates of the same requests (comma list; empty = none)")
    ap.add_argument("--cs-sat-rate", type=float, default=50000.0,
                    help="arrival rate of a last serving run that saturates the loop (0 = skip)")
    ap.add_argument("--cs-budget", type=int, default=32768, help="serving memory budget, MiB")
    ap.add_argument("--pool-bricks", type=int, default=0, help="brick slots to reserve (0 = default)")
    ap.add_argument("--tuning", default="",
                    help="launch tuning of the headline view as comma-separated rkf_batch_tuning fields "
                         "(tile_w,tile_h,step_budget,...); skips the autotuner")
    ap.add_argument("--no-reference-pool", action="store_true",
                    help="keep no AoS reference pool (implies --no-plain; smaller device footprint)")
    ap.add_argument("--report", default="", choices=["", "precision"],
                    help="print a study instead of the benchmark line")
    return ap.parse_args()


def spec_of(name):
    return scenes.SCENE_LARGE if name == "large" else scenes.SCENE_SMALL


def camera_for(spec, w, h, rank):
    # seeded pose inside the cube for the large scene (the outside view of a
    # 256 m cube is mostly sky); outside for the small scene
    if spec is scenes.SCENE_LARGE:
        return scenes.seeded_camera(spec, w, h, seed=100 + rank, inside=True, distance=spec.cube * 0.18)
    return scenes.seeded_camera(spec, w, h, seed=11 + rank)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed regions:
    polled every 20 ms from before the first timed region to after the last;
    the summary counts the samples taken inside a window()."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []    # (arrival time, csv line)
        self.windows = []  # timed regions (perf_counter start, end)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the first query takes a while: start timing once samples flow
            t_end = time.perf_counter() + 5.0
            while not self.lines and time.perf_counter() < t_end and self.proc.poll() is None:
                time.sleep(0.005)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.perf_counter(), ln.strip()))

    @contextlib.contextmanager
    def window(self):
        t0 = time.perf_counter()
        try:
            yield
        finally:
            self.windows.append((t0, time.perf_counter()))

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # a line arrives up to one query (a few ms) after its sample was taken
        inside = [ln for t, ln in self.lines
                  if not self.windows or any(a <= t <= b + 0.02 for a, b in self.windows)]
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist  # plumbing only: barrier and max over ranks
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def dist_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def job_mrays(dist, world: int, rays_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job rate of replicas: every rank marches rays_per_rank rays per
    step; the job takes as long as its slowest rank."""
    return world * rays_per_rank * steps / dist_max(dist, seconds) / 1e6


def oracle_scene_from_ctx(ctx, oracle):
    info = ctx.info()
    words = ctx.export_pool(0, info["pool_bricks_used"])
    idx = ctx.export_index()
    obj = ctx.object(0)
    return oracle.Scene([obj], pool_words=words, top=idx["top"], leaves=idx["leaves"],
                        obj_top_info=idx["obj_top_info"])


def sample_rows(h, n):
    n = max(1, min(n, h))
    return [int(r) for r in np.linspace(0, h - 1, n).round()]


def cpu_march_rate(oracle, sc, cam, p, w, h, rows, threads):
    """Mrays/s of the FP32 restatement over the given rows (all threads)."""
    t0 = time.perf_counter()
    n = 0
    for r in rows:
        oracle.march(sc, cam, p, w, h, threads=threads, rows=(r, r + 1))
        n += w
    dt = time.perf_counter() - t0
    return n / dt / 1e6, n, dt


def sector_stats(oracle, sc, cam, p, w, h, rows, threads):
    tot = {"sectors": 0, "index_sectors": 0, "dist_sectors": 0, "mat_sectors": 0, "steps": 0, "rays": 0,
           "hits": 0}
    for r in rows:
        o = oracle.march(sc, cam, p, w, h, threads=threads, rows=(r, r + 1), count_sectors=True)
        for k in ("sectors", "index_sectors", "dist_sectors", "mat_sectors", "steps"):
            tot[k] += o["stats"][k]
        tot["rays"] += w
        tot["hits"] += int((o["flags"] & 1).sum())
    return tot


def load_traffic(workload):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return d.get(workload)
    except Exception:
        return None


def run_reference(args, world, rank, dist):
    """CPU implementation of the reference algorithm, bounded sample."""
    if rank != 0:
        return
    from oracle import binding as oracle
    spec = spec_of(args.scene)
    w, h = args.width, args.height
    threads = os.cpu_count() or 1
    prims = scenes.make_prims(spec)
    vp = scenes.voxelize_params(spec, prims)
    t0 = time.perf_counter()
    if args.scene == "small":
        v = oracle.Voxelized(prims, vp, threads=threads)
        sc = oracle.Scene([v.gpu_object()], pool_words=v.words, brick_maps=v.map)
    else:
        # the CPU restatement of the voxelizer, into a two-level index (a flat
        # brick map of this grid would take 17.6 GB); untimed set-up
        v = oracle.SparseVoxelized(prims, vp, threads=threads)
        sc = v.scene()
    build_s = time.perf_counter() - t0
    cam = camera_for(spec, w, h, 0)
    p = scenes.march_params(spec)
    rows = sample_rows(h, args.cpu_rows)
    oracle.march(sc, cam, p, w, h, threads=threads, rows=(rows[0], rows[0] + 1))  # warm
    rates = []
    for _ in range(max(1, args.steps)):
        r, n, dt = cpu_march_rate(oracle, sc, cam, p, w, h, rows, threads)
        rates.append(r)
        if sum(rates) and len(rates) * dt > 120:
            break
    value = float(np.median(rates))
    sample = f"{len(rows)} rows x {w} px of the {w}x{h} view per step ({len(rows) * w} rays)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": len(rates), "warmup": args.warmup, "ms_per_step": 1e3 * len(rows) * w / (value * 1e6),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded primitives voxelized on the fly)",
        "config": {"workload": f"{spec.name} {w}x{h} primary view", "rays_per_step": len(rows) * w,
                   "scene_build_s": build_s, "scene_build": "CPU restatement of the voxelizer (untimed)"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def build_batching(ctx, spec, prims, p, n_views, seed):
    """Views of uneven size plus their shadow / AO ray batches, on the device."""
    import ctypes as C

    from rkifield_b200 import cudart, workloads
    views = workloads.make_views(spec, prims, n_views, seed)
    vs = (abi.rkf_view * len(views))()
    keep = []
    n_primary = 0
    for i, v in enumerate(views):
        g = cudart.device_gbuffer(v.width * v.height)
        keep.append(g)
        vs[i].camera = v.cam
        vs[i].width, vs[i].height = v.width, v.height
        for k, a in g.items():
            setattr(vs[i].out, k, a.ptr)
        vs[i].out.mem = abi.RKF_MEM_DEVICE
        n_primary += v.width * v.height
    abi.check(ctx.lib.rkf_march_batch(ctx.h, vs, len(views), None, 0, C.byref(p), None), "batch primaries")
    rng = np.random.default_rng(seed + 1)
    batches = (abi.rkf_ray_batch * (2 * len(views)))()
    n_live = 0
    n_slots = 0
    for i, v in enumerate(views):
        npx = v.width * v.height
        g = keep[i]
        target = np.array(v.cam.position[:3], np.float64) + 8.0 * np.array(v.cam.forward[:3], np.float64)
        lights = (target[None] + rng.uniform(-10, 10, (4, 3)) + np.array([0.0, 8.0, 0.0])).astype(np.float32)
        arrs = [cudart.DeviceArray(3 * 4 * npx, np.float32), cudart.DeviceArray(3 * 4 * npx, np.float32),
                cudart.DeviceArray(4 * npx, np.float32), cudart.DeviceArray(3 * 8 * npx, np.float32),
                cudart.DeviceArray(3 * 8 * npx, np.float32), cudart.DeviceArray(8 * npx, np.float32)]
        keep.append(arrs)
        hits = C.c_uint32()
        gbs = abi.rkf_gbuffer()
        gbs.t, gbs.normal, gbs.flags, gbs.mem = g["t"].ptr, g["normal"].ptr, g["flags"].ptr, abi.RKF_MEM_DEVICE
        abi.check(ctx.lib.rkf_secondary_rays(ctx.h, C.byref(v.cam), v.width, v.height, C.byref(gbs),
                                             lights.ctypes.data, 4, 8, 1.0, seed * 1000 + i,
                                             *[a.ptr for a in arrs], C.byref(hits), None), "secondary rays")
        n_live += hits.value * 12
        for j, (o, d, t, nper, mode) in enumerate(((arrs[0], arrs[1], arrs[2], 4, abi.RKF_TRACE_SHADOW),
                                                   (arrs[3], arrs[4], arrs[5], 8, abi.RKF_TRACE_ANY))):
            out = {"t": cudart.DeviceArray(nper * npx, np.float32), "flags": cudart.DeviceArray(nper * npx, np.uint16)}
            keep.append(out)
            b = batches[2 * i + j]
            b.origins, b.dirs, b.tmax, b.n, b.mode = o.ptr, d.ptr, t.ptr, nper * npx, mode
            b.out.t, b.out.flags, b.out.mem = out["t"].ptr, out["flags"].ptr, abi.RKF_MEM_DEVICE
            n_slots += nper * npx
    return {"views": views, "vs": vs, "batches": batches, "keep": keep, "n_primary": n_primary,
            "n_secondary_live": n_live, "n_secondary_slots": n_slots}


def run_batching(ctx, spec, prims, p, args, stream):
    import ctypes as C

    from rkifield_b200 import cudart
    wl = build_batching(ctx, spec, prims, p, args.cb_views, seed=300)
    nv = len(wl["views"])
    vs, bs = wl["vs"], wl["batches"]
    # autotune on a sample: the first eighth of the views and their secondaries
    ns = max(1, nv // 8)
    tu = abi.rkf_batch_tuning()
    t0 = time.perf_counter()
    abi.check(ctx.lib.rkf_autotune(ctx.h, vs, ns, bs, 2 * ns, C.byref(p), C.byref(tu)), "autotune")
    tune_s = time.perf_counter() - t0

    def timed(fn, steps):
        fn()
        stream.synchronize()
        ms = []
        for _ in range(steps):
            a, b = cudart.Event(), cudart.Event()
            a.record(stream)
            fn()
            b.record(stream)
            stream.synchronize()
            ms.append(a.elapsed_ms(b))
        return ms

    def batched():
        abi.check(ctx.lib.rkf_march_batch_async(ctx.h, vs, nv, bs, 2 * nv, C.byref(p), None, stream.ptr), "batch")

    def per_request(plain):
        for i in range(nv):
            v = vs[i]
            fn = ctx.lib.rkf_march_plain_async if plain else ctx.lib.rkf_march_async
            abi.check(fn(ctx.h, C.byref(v.camera), C.byref(p), v.width, v.height, C.byref(v.out), stream.ptr),
                      "view")
        for j in range(2 * nv):
            b = bs[j]
            if plain:
                abi.check(ctx.lib.rkf_trace_rays_plain_async(ctx.h, b.origins, b.dirs, b.tmax, b.n, b.mode,
                                                             C.byref(p), C.byref(b.out), stream.ptr), "rays")
            else:
                abi.check(ctx.lib.rkf_march_batch_async(ctx.h, None, 0, C.byref(b), 1, C.byref(p), None,
                                                        stream.ptr), "rays")

    steps = args.cb_steps
    mb = timed(batched, steps)
    # the same batch captured once as a CUDA graph and replayed
    from rkifield_b200.engine import BatchGraph
    graph = BatchGraph(ctx, vs, bs, p)
    try:
        mg = timed(lambda: graph.launch(stream.ptr), steps)
    finally:
        stream.synchronize()
        graph.close()
    mp = timed(lambda: per_request(True), max(1, steps - 1))
    mf = timed(lambda: per_request(False), max(1, steps - 1))
    rays = wl["n_primary"] + wl["n_secondary_live"]
    val = lambda ms: rays / (np.mean(ms) / 1e3) / 1e6  # noqa: E731
    return {"views": nv, "primary_rays": wl["n_primary"], "secondary_rays_live": wl["n_secondary_live"],
            "secondary_ray_slots": wl["n_secondary_slots"],
            "tuning": {"tile": [tu.tile_w, tu.tile_h], "compact_interval": tu.compact_interval,
                       "step_budget": tu.step_budget, "refill_idle": tu.refill_idle,
                       "probe_in_run": tu.probe_in_run, "no_empty_path": tu.no_empty_path,
                       "threads_per_block": tu.threads_per_block, "tune_s": tune_s},
            "batched": {"value": val(mb), "unit": "Mrays/s", "ms": float(np.mean(mb)), "launches": 1},
            "batched_graph": {"value": val(mg), "unit": "Mrays/s", "ms": float(np.mean(mg)), "launches": 1},
            "plain_per_request": {"value": val(mp), "unit": "Mrays/s", "ms": float(np.mean(mp)),
                                  "launches": 3 * nv},
            "b200_per_request": {"value": val(mf), "unit": "Mrays/s", "ms": float(np.mean(mf)),
                                 "launches": 3 * nv},
            "vs_plain": val(mb) / val(mp)}


def _pinned_copy(arrs, keep):
    """Copies of the given arrays in one page-locked block (async copies)."""
    from rkifield_b200 import cudart
    total = sum(a.nbytes for a in arrs) + 256 * len(arrs)
    blk = cudart.PinnedArray(total, np.uint8)
    keep.append(blk)
    out, off = [], 0
    for a in arrs:
        v = blk.array[off:off + a.nbytes].view(a.dtype)
        v[:] = a.ravel()
        out.append(v)
        off += (a.nbytes + 255) // 256 * 256
    return out


def warm_serving(local):
    """Untimed: a short serving session on the small scene (every request
    kind and a few edits), so the first launch of each serving-path kernel,
    with its module load, happens before the timed runs."""
    from rkifield_b200 import engine, workloads
    from rkifield_b200.engine import Context, Server
    spec = scenes.SCENE_SMALL
    prims = scenes.make_prims(spec)
    reqs = workloads.make_request_stream(spec, prims, 40, seed=7, rate_hz=1e6, edit_every=8,
                                         max_rays=4096, max_points=4096, render_area=(64 ** 2, 128 ** 2))
    ctx = Context(device=local, pool_capacity=65536)
    keep = []
    try:
        ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
        srv = Server(ctx, scenes.march_params(spec))
        tks = []
        for r in reqs:
            if r.kind == 0:
                o = engine.render_out(r.width * r.height)
                keep.append(o)
                tks.append(srv.submit_render(r.cam, r.width, r.height, o))
            elif r.kind == 1:
                o = engine.rays_out(r.n, 0)
                keep.append((r, o))
                tks.append(srv.submit_rays(r.o, r.d, r.tmax, 0, o))
            elif r.kind == 2:
                o = engine.points_out(r.n)
                keep.append((r, o))
                tks.append(srv.submit_points(r.points, o))
            else:
                tks.append(srv.submit_edit(r.edit))
        for tk in tks:
            while srv.poll(tk, 100000) is None:
                pass
        srv.stop()
    finally:
        ctx.close()


def run_serving(args, spec, prims, p, local, rates, with_plain=True):
    """Poisson request stream through the serving loop at each offered rate
    (the same requests, arrivals scaled), vs plain per-request launches of
    the same requests (one at a time in arrival order; their service times
    are measured once, and each rate's latencies follow from its arrivals)."""
    from rkifield_b200 import workloads
    base = workloads.make_request_stream(spec, prims, args.cs_requests, seed=500, rate_hz=args.cs_rate)
    keep = []
    bufs = _serving_buffers(base, keep)
    plain = _serving_plain(args, spec, prims, p, local, base, bufs) if with_plain else None
    out = {"requests": len(base), "rays": sum(r.n for r in base if r.kind in (0, 1)),
           "points": sum(r.n for r in base if r.kind == 2), "edits": sum(1 for r in base if r.kind == 3),
           "by_rate": []}
    for rate in rates:
        scale = args.cs_rate / rate
        reqs = [dataclasses.replace(r, arrival_s=r.arrival_s * scale) for r in base]
        served = _serving_served(args, spec, prims, p, local, reqs, bufs)
        row = {"rate_hz": rate, "served": served}
        if plain is not None:
            lat_p = _fifo_latency(reqs, plain["service_s"])
            row["plain_latency_ms"] = {"p50": float(np.percentile(lat_p, 50)), "p99": float(np.percentile(lat_p, 99))}
            row["vs_plain"] = served["value"] / plain["value"]
        out["by_rate"].append(row)
    if plain is not None:
        out["plain_per_request"] = {k: v for k, v in plain.items() if k != "service_s"}
    return out


def _fifo_latency(reqs, service):
    """Latencies (ms) of a single FIFO server with the given service times."""
    done, lat = 0.0, []
    for r, s in zip(reqs, service):
        start = max(done, r.arrival_s)
        done = start + s
        lat.append((done - r.arrival_s) * 1e3)
    return lat


def _serving_buffers(reqs, keep):
    """Page-locked inputs and outputs for every request."""
    from rkifield_b200 import engine
    bufs = []
    for r in reqs:
        if r.kind == 0:
            o = engine.render_out(r.width * r.height)
            names = list(o)
            pin = _pinned_copy([o[k] for k in names], keep)
            bufs.append((None, dict(zip(names, pin))))
        elif r.kind == 1:
            ins = _pinned_copy([r.o, r.d, r.tmax], keep)
            o = engine.rays_out(r.n, 0)
            names = list(o)
            bufs.append((ins, dict(zip(names, _pinned_copy([o[k] for k in names], keep)))))
        elif r.kind == 2:
            ins = _pinned_copy([r.points], keep)
            o = engine.points_out(r.n)
            names = list(o)
            bufs.append((ins, dict(zip(names, _pinned_copy([o[k] for k in names], keep)))))
        else:
            bufs.append((None, None))
    return bufs


def _serving_served(args, spec, prims, p, local, reqs, bufs):
    """One serving session over the requests at their arrival times."""
    from rkifield_b200.engine import Context, RkfError, Server
    total_rays = sum(r.n for r in reqs if r.kind in (0, 1))
    total_pts = sum(r.n for r in reqs if r.kind == 2)
    ctx = Context(device=local, pool_capacity=LARGE_POOL, mem_budget_bytes=args.cs_budget << 20,
                  max_inflight=1024)
    ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
    srv = Server(ctx, p)
    t0 = time.perf_counter()
    i, live, res, busy = 0, {}, [None] * len(reqs), 0
    submit_wall = [0.0] * len(reqs)
    while i < len(reqs) or live:
        now = time.perf_counter() - t0
        while i < len(reqs) and reqs[i].arrival_s <= now:
            r = reqs[i]
            ins, out = bufs[i]
            try:
                if r.kind == 0:
                    tk = srv.submit_render(r.cam, r.width, r.height, out)
                elif r.kind == 1:
                    tk = srv.submit_rays(ins[0], ins[1], ins[2], 0, out)
                elif r.kind == 2:
                    tk = srv.submit_points(ins[0], out)
                else:
                    tk = srv.submit_edit(r.edit)
            except RkfError as e:
                if e.status != abi.RKF_BUSY:
                    raise
                busy += 1
                break  # admission refused: retry this request on the next pass
            submit_wall[i] = time.perf_counter() - t0
            live[tk] = i
            i += 1
        # collect in admission order up to the first unfinished request; the
        # results carry the loop's own completion times, so collecting late
        # does not change a latency, and the host spends its time submitting
        for tk in list(live):
            rr = srv.poll(tk, 0)
            if rr is None:
                break
            res[live.pop(tk)] = rr
        if live and (i >= len(reqs) or reqs[i].arrival_s > time.perf_counter() - t0):
            time.sleep(20e-6)
    wall = time.perf_counter() - t0
    srv.stop()
    ctx.close()
    # latency = admission delay (arrival -> accepted) + loop latency (accepted -> done)
    lat = np.array([(submit_wall[k] - reqs[k].arrival_s) * 1e3 + (res[k]["done_us"] - res[k]["submit_us"]) / 1e3
                    for k in range(len(reqs))])
    return {"value": total_rays / wall / 1e6, "unit": "Mrays/s", "points_per_s": total_pts / wall,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "busy_retries": busy, "wall_s": wall, "offered_s": reqs[-1].arrival_s}


def _serving_plain(args, spec, prims, p, local, reqs, bufs):
    """Each request through its own launches, one at a time in arrival order."""
    import ctypes as C

    from rkifield_b200 import cudart, engine
    from rkifield_b200.engine import Context
    total_rays = sum(r.n for r in reqs if r.kind in (0, 1))
    total_pts = sum(r.n for r in reqs if r.kind == 2)

    # ---- plain: one launch per request, in arrival order, one at a time --------
    # device buffers are allocated once (the largest request); each request
    # copies its inputs in from page-locked memory, launches, copies back
    ctx = Context(device=local, pool_capacity=LARGE_POOL)
    ctx.voxelize(prims, scenes.voxelize_params(spec, prims))
    stream = cudart.Stream()
    max_rays = max([r.n for r in reqs if r.kind == 1] + [1])
    dev_in = [cudart.DeviceArray(3 * max_rays, np.float32), cudart.DeviceArray(3 * max_rays, np.float32),
              cudart.DeviceArray(max_rays, np.float32)]
    ray_planes = engine.rays_out(max_rays, 0)
    dev_out = {kk: cudart.DeviceArray(v.size, v.dtype) for kk, v in ray_planes.items()}
    hits = abi.rkf_hits()
    for kk, v in dev_out.items():
        setattr(hits, kk, v.ptr)
    hits.mem = abi.RKF_MEM_DEVICE
    service = []
    for k, r in enumerate(reqs):
        ins, out = bufs[k]
        a = time.perf_counter()
        if r.kind == 0:
            ctx.march(r.cam, p, r.width, r.height, out=out, plain=True)
        elif r.kind == 1:
            n = r.n
            for dv, hv in zip(dev_in, ins):
                dv.upload(hv, stream)
            abi.check(ctx.lib.rkf_trace_rays_plain_async(ctx.h, dev_in[0].ptr, dev_in[1].ptr, dev_in[2].ptr, n, 0,
                                                         C.byref(p), C.byref(hits), stream.ptr), "plain rays")
            for kk, v in out.items():
                dev_out[kk].download_into(v, stream)
            stream.synchronize()
        elif r.kind == 2:
            d, g, m = ctx.query_points(ins[0])
            out["dist"][:], out["grad"][:], out["material"][:] = d, g, m
        else:
            ctx.edit(r.edit)
        service.append(time.perf_counter() - a)
    ctx.close()
    plain_wall = sum(service)
    lat_p = _fifo_latency(reqs, service)
    return {"value": total_rays / plain_wall / 1e6, "unit": "Mrays/s", "points_per_s": total_pts / plain_wall,
            "latency_ms_at_base_rate": {"p50": float(np.percentile(lat_p, 50)),
                                        "p99": float(np.percentile(lat_p, 99))},
            "service_s": service}


def run_precision_report(args):
    """Storage precision study on the small scene: per-ray error of the march
    over f32 / f16 / u8 planes against the FP64 march over the analytic
    voxel values (same control flow), 1920x1080 primary rays plus AO rays."""
    import ctypes as C

    from oracle import binding as oracle
    from rkifield_b200 import cudart
    from rkifield_b200.engine import Context
    spec = scenes.SCENE_SMALL
    prims = scenes.make_prims(spec)
    vp = scenes.voxelize_params(spec, prims)
    w, h = args.width, args.height
    cam = scenes.seeded_camera(spec, w, h, seed=11)
    p = scenes.march_params(spec)
    vs = spec.voxel_size
    threads = os.cpu_count() or 1
    v = oracle.Voxelized(prims, vp, threads=threads)
    f64 = oracle.voxel_values_f64(prims, vp, v.map, v.n_bricks, threads)
    w0 = v.words[0::2]
    mat = (((w0 >> 16) & 0x3F) | (((w0 >> 22) & 0x3F) << 6)).astype(np.uint16)
    blend = (v.words[1::2] >> 24).astype(np.uint8)
    sc64 = oracle.Scene([v.gpu_object()], brick_maps=v.map, mat_plane=mat, blend_plane=blend,
                        precision=oracle.PRECISION_F64, dist_f64=f64)
    t0 = time.perf_counter()
    ref = oracle.march(sc64, cam, p, w, h, fp64=True, threads=threads, with_margin=True)
    oracle_s = time.perf_counter() - t0
    hit64 = (ref["flags"] & 1) != 0
    n64 = ref["normal64"].reshape(-1, 3)
    report = {"scene": spec.name, "view": f"{w}x{h}", "rays": w * h, "fp64_hit_fraction": float(hit64.mean()),
              "fp64_oracle_s": oracle_s, "precisions": {}}
    ao_ref = None
    # u8: codes rounded toward zero (never overstating |d|) and to nearest
    for name, prec, rnd in (("f32", "f32", 0), ("f16", "f16", 0), ("u8", "u8", 0), ("u8_nearest", "u8", 1)):
        ctx = Context(pool_capacity=v.n_bricks + 1024, precision=prec, keep_reference_pool=False, u8_round=rnd)
        ctx.voxelize(prims, vp)
        g = ctx.march(cam, p, w, h)
        hit = (g["flags"] & 1) != 0
        both = hit & hit64
        # grazing: a decision of the FP64 march within 1e-3 voxel of its threshold,
        # or a hit whose ray meets the surface at under ~3 degrees
        graze = ref["margin"] < 1e-3 * vs
        dirs_dot = None
        nonz = both & ~graze
        dt = np.abs(g["t"][nonz].astype(np.float64) - ref["t64"][nonz]) / vs
        ng = g["normal"].reshape(-1, 3)[nonz].astype(np.float64)
        cosang = np.clip(np.sum(ng * n64[nonz], axis=1) / np.maximum(
            np.linalg.norm(ng, axis=1) * np.linalg.norm(n64[nonz], axis=1), 1e-300), -1.0, 1.0)
        ang = np.arccos(cosang)
        del dirs_dot
        # the same error on the rays none of whose FP64 decisions lies within
        # m voxels of its threshold: a code error of m can flip no decision
        # there, so what remains is the values' own error, not a step's jump
        by_margin = {}
        for m in (0.0118, 0.0236, 0.05):
            keep = both & (ref["margin"] >= m * vs)
            dm = np.abs(g["t"][keep].astype(np.float64) - ref["t64"][keep]) / vs
            by_margin[str(m)] = {"hit_rays_kept": float(keep.sum() / max(1, both.sum())),
                                 "p99": float(np.percentile(dm, 99)) if dm.size else None,
                                 "mean": float(dm.mean()) if dm.size else None,
                                 "within_0.01_voxel": float((dm <= 0.01).mean()) if dm.size else None}
        entry = {"dt_voxels_by_decision_margin": by_margin,
                 "hit_agreement": float((hit == hit64).mean()),
                 "hit_agreement_non_grazing": float((hit == hit64)[~graze].mean()),
                 "material_agreement": float((g["material"][both] == ref["material"][both]).mean()) if both.any() else None,
                 "grazing_fraction": float(graze.mean()),
                 "dt_voxels": {"max": float(dt.max()), "p99": float(np.percentile(dt, 99)), "mean": float(dt.mean())},
                 "normal_rad": {"max": float(ang.max()), "p99": float(np.percentile(ang, 99)), "mean": float(ang.mean())},
                 "within_0.01_voxel": float((dt <= 0.01).mean()),
                 "bytes_per_voxel_distance": {"f32": 4, "f16": 2, "u8": 1}[prec]}
        # AO rays (any hit, 1 m) from the FP64 primary hits, traced through each plane
        if ao_ref is None:
            dev = cudart.device_gbuffer(w * h)
            for k in ("t", "normal", "flags"):
                dev[k].upload(g[k] if k != "t" else np.where(hit64, ref["t64"], 3.4e38).astype(np.float32))
            dev["flags"].upload(np.where(hit64, 1, 0).astype(np.uint16))
            dev["normal"].upload(n64.astype(np.float32).ravel())
            rays = [cudart.DeviceArray(3 * 8 * w * h, np.float32), cudart.DeviceArray(3 * 8 * w * h, np.float32),
                    cudart.DeviceArray(8 * w * h, np.float32)]
            gb = abi.rkf_gbuffer()
            gb.t, gb.normal, gb.flags, gb.mem = dev["t"].ptr, dev["normal"].ptr, dev["flags"].ptr, abi.RKF_MEM_DEVICE
            nh = C.c_uint32()
            abi.check(ctx.lib.rkf_secondary_rays(ctx.h, C.byref(cam), w, h, C.byref(gb), None, 0, 8, 1.0, 7,
                                                 None, None, None, rays[0].ptr, rays[1].ptr, rays[2].ptr,
                                                 C.byref(nh), None), "ao rays")
            ao_o, ao_d, ao_t = (r.download() for r in rays)
            live = ao_t > 0
            ao_o, ao_d, ao_t = ao_o.reshape(-1, 3)[live], ao_d.reshape(-1, 3)[live], ao_t[live]
            ao_ref = oracle.trace(sc64, ao_o.ravel(), ao_d.ravel(), ao_t, abi.RKF_TRACE_ANY, p, fp64=True,
                                  threads=threads, with_margin=True)
        ao = ctx.trace(ao_o, ao_d, ao_t, abi.RKF_TRACE_ANY, p)
        ag = (ao["flags"] & 1) == (ao_ref["flags"] & 1)
        entry["ao_rays"] = int(ao_t.size)
        entry["ao_occlusion_agreement"] = float(ag.mean())
        entry["ao_occlusion_agreement_non_grazing"] = float(ag[ao_ref["margin"] >= 1e-3 * vs].mean())
        report["precisions"][name] = entry
        ctx.close()
    print(json.dumps({"report": "precision", **report}), flush=True)


def _view_dirs(cam, w, h):
    """Unit primary-ray directions of a view (float64, ray_march.wgsl:1046-1053)."""
    px, py = np.meshgrid(np.arange(w, dtype=np.float64), np.arange(h, dtype=np.float64))
    u, v = (px.ravel() + 0.5) / w, (py.ravel() + 0.5) / h
    fwd, right, up = (np.array(x[:3], np.float64) for x in (cam.forward, cam.right, cam.up))
    d = fwd[None] + (2 * u - 1)[:, None] * right[None] + (1 - 2 * v)[:, None] * up[None]
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def _error_entry(g, ref, dirs, vs):
    """Per-view error of a device march against the FP64 march, with the
    grazing rays of the parity rule set aside: an FP64 decision within 1e-3
    voxel of its threshold, a hit at under 0.05 of normal incidence, or a
    hit/miss the device (FP32) and FP64 marches disagree on."""
    hit = (g["flags"] & 1) != 0
    hit64 = (ref["flags"] & 1) != 0
    n64 = ref["normal64"].reshape(-1, 3)
    cosi = np.abs(np.sum(dirs * n64, axis=1))
    graze = (ref["margin"] < 1e-3 * vs) | (hit64 & (cosi < 0.05)) | (hit != hit64)
    both = hit & hit64 & ~graze
    dt = np.abs(g["t"][both].astype(np.float64) - ref["t64"][both]) / vs
    ng = g["normal"].reshape(-1, 3)[both].astype(np.float64)
    cosang = np.clip(np.sum(ng * n64[both], axis=1) / np.maximum(
        np.linalg.norm(ng, axis=1) * np.linalg.norm(n64[both], axis=1), 1e-300), -1.0, 1.0)
    ang = np.arccos(cosang)
    q = lambda a, f: float(f(a)) if a.size else None  # noqa: E731
    return {"rays": int(hit.size), "fp64_hits": int(hit64.sum()), "grazing_fraction": float(graze.mean()),
            "hit_agreement": float((hit == hit64).mean()),
            "hit_agreement_non_grazing": float((hit == hit64)[~graze].mean()),
            "material_agreement": float((g["material"][both] == ref["material"][both]).mean()) if both.any() else None,
            "dt_voxels": {"max": q(dt, np.max), "p99": q(dt, lambda a: np.percentile(a, 99)), "mean": q(dt, np.mean)},
            "within_0.01_voxel": q(dt, lambda a: (a <= 0.01).mean()),
            "normal_rad": {"max": q(ang, np.max), "p99": q(ang, lambda a: np.percentile(a, 99)),
                           "mean": q(ang, np.mean)}}


def run_precision_report_large(args):
    """FP64 error of the large scene's f16 march: the headline view at
    1920x1080 and 960x540, three views of the batching workload (smallest,
    median, largest) and 20,000 of their soft-shadow and AO rays, against the
    FP64 march over FP64 voxel values at the same voxel centres."""
    import ctypes as C

    from oracle import binding as oracle
    from rkifield_b200 import cudart, workloads
    from rkifield_b200.engine import Context
    spec = scenes.SCENE_LARGE
    prims = scenes.make_prims(spec)
    vp = scenes.voxelize_params(spec, prims)
    p = scenes.march_params(spec)
    vs = spec.voxel_size
    threads = os.cpu_count() or 1
    ctx = Context(pool_capacity=LARGE_POOL, keep_reference_pool=False)
    ctx.voxelize(prims, vp)
    idx = ctx.export_index()
    t0 = time.perf_counter()
    bxyz, slots = oracle.index_bricks(idx["top"], idx["leaves"], idx["obj_top_info"])
    n_slots = int(slots.max()) + 1
    pl = ctx.export_planes(0, n_slots)
    f64 = oracle.voxel_values_f64_bricks(prims, vp, bxyz, slots, n_slots, threads)
    values_s = time.perf_counter() - t0
    obj = ctx.object(0)
    sc64 = oracle.Scene([obj], top=idx["top"], leaves=idx["leaves"], obj_top_info=idx["obj_top_info"],
                        mat_plane=pl["mat"], blend_plane=pl["blend"], precision=oracle.PRECISION_F64, dist_f64=f64)
    report = {"scene": spec.name, "bricks": int(slots.size), "fp64_values_s": values_s, "views": {}}
    views = [("headline 1920x1080", camera_for(spec, 1920, 1080, 0), 1920, 1080),
             ("headline 960x540", camera_for(spec, 960, 540, 0), 960, 540)]
    cb = workloads.make_views(spec, prims, 64, seed=300)
    order = np.argsort([v.width * v.height for v in cb], kind="stable")
    for name, i in (("batch smallest", order[0]), ("batch median", order[len(order) // 2]),
                    ("batch largest", order[-1])):
        v = cb[i]
        views.append((f"{name} {v.width}x{v.height}", v.cam, v.width, v.height))
    cb_gbufs = []
    for name, cam, w, h in views:
        t1 = time.perf_counter()
        g = ctx.march(cam, p, w, h)
        ref = oracle.march(sc64, cam, p, w, h, fp64=True, threads=threads, with_margin=True)
        e = _error_entry(g, ref, _view_dirs(cam, w, h), vs)
        e["fp64_march_s"] = time.perf_counter() - t1
        report["views"][name] = e
        if name.startswith("batch"):
            cb_gbufs.append((cam, w, h, g))
        print(json.dumps({name: e}), file=sys.stderr, flush=True)
    # secondary rays of the three batch views, through the device march and FP64
    rng = np.random.default_rng(17)
    sec = {"shadow": [], "ao": []}
    for i, (cam, w, h, g) in enumerate(cb_gbufs):
        npx = w * h
        dev = cudart.device_gbuffer(npx)
        for k in ("t", "normal", "flags"):
            dev[k].upload(g[k])
        target = np.array(cam.position[:3], np.float64) + 8.0 * np.array(cam.forward[:3], np.float64)
        lights = (target[None] + rng.uniform(-10, 10, (4, 3)) + np.array([0.0, 8.0, 0.0])).astype(np.float32)
        arrs = [cudart.DeviceArray(3 * 4 * npx, np.float32), cudart.DeviceArray(3 * 4 * npx, np.float32),
                cudart.DeviceArray(4 * npx, np.float32), cudart.DeviceArray(3 * 8 * npx, np.float32),
                cudart.DeviceArray(3 * 8 * npx, np.float32), cudart.DeviceArray(8 * npx, np.float32)]
        gb = abi.rkf_gbuffer()
        gb.t, gb.normal, gb.flags, gb.mem = dev["t"].ptr, dev["normal"].ptr, dev["flags"].ptr, abi.RKF_MEM_DEVICE
        nh = C.c_uint32()
        abi.check(ctx.lib.rkf_secondary_rays(ctx.h, C.byref(cam), w, h, C.byref(gb), lights.ctypes.data, 4, 8, 1.0,
                                             300 * 1000 + i, *[a.ptr for a in arrs], C.byref(nh), None), "secondary")
        for key, (o, d, t) in (("shadow", arrs[0:3]), ("ao", arrs[3:6])):
            tm = t.download()
            live = np.nonzero(tm > 0)[0]
            sel = live if live.size <= 3400 else np.sort(rng.choice(live, 3400, replace=False))
            sec[key].append((o.download().reshape(-1, 3)[sel], d.download().reshape(-1, 3)[sel], tm[sel]))
    for key, mode in (("shadow", abi.RKF_TRACE_SHADOW), ("ao", abi.RKF_TRACE_ANY)):
        o = np.concatenate([a[0] for a in sec[key]])
        d = np.concatenate([a[1] for a in sec[key]])
        tm = np.concatenate([a[2] for a in sec[key]])
        got = ctx.trace(o, d, tm, mode, p)
        ref = oracle.trace(sc64, o.ravel(), d.ravel(), tm, mode, p, fp64=True, threads=threads, with_margin=True)
        ok = ref["margin"] >= 1e-3 * vs
        ent = {"rays": int(tm.size), "grazing_fraction": float((~ok).mean()),
               "occlusion_agreement": float(((got["flags"] & 1) == (ref["flags"] & 1)).mean()),
               "occlusion_agreement_non_grazing": float(((got["flags"] & 1) == (ref["flags"] & 1))[ok].mean())}
        if mode == abi.RKF_TRACE_SHADOW:
            ds = np.abs(got["t"].astype(np.float64) - ref["t64"])[ok]
            ent["shadow_factor_abs_err"] = {"max": float(ds.max()), "p99": float(np.percentile(ds, 99)),
                                            "mean": float(ds.mean())}
        report["secondary_" + key] = ent
    ctx.close()
    print(json.dumps({"report": "precision_large", **report}), flush=True)


def time_view(ctx, cam, p, w, h, stream, steps, plain=False):
    """Mean CUDA-event ms of one view march (untimed warm-up first)."""
    from rkifield_b200 import cudart
    g = cudart.device_gbuffer(w * h)
    gp = cudart.gbuffer_ptrs(g)
    ctx.march_async(cam, p, w, h, gp, stream.ptr, plain=plain)
    ms = []
    for _ in range(steps):
        a, b = cudart.Event(), cudart.Event()
        a.record(stream)
        ctx.march_async(cam, p, w, h, gp, stream.ptr, plain=plain)
        b.record(stream)
        stream.synchronize()
        ms.append(a.elapsed_ms(b))
    return float(np.mean(ms))


def run_extras(args, spec, prims, p, ctx, stream):
    """Secondary figures: the 960x540 view, and the headline view over the f32
    and u8 distance planes (same scene, separate contexts)."""
    from rkifield_b200.engine import Context
    out = {}
    w, h = 960, 540
    cam = camera_for(spec, w, h, 0)
    b = time_view(ctx, cam, p, w, h, stream, 5)
    v = {"b200_mrays": w * h / b / 1e3, "b200_ms": b}
    if not args.no_plain:
        pl = time_view(ctx, cam, p, w, h, stream, 2, plain=True)
        v.update(plain_mrays=w * h / pl / 1e3, plain_ms=pl, vs_plain=pl / b)
    out["view_960x540"] = v
    prec = {}
    cam = camera_for(spec, args.width, args.height, 0)
    n = args.width * args.height
    # the headline view under the shader's other strategies (the runtime binds
    # tile lists every frame, so its shader marches with the tiled one)
    from rkifield_b200 import engine
    ctx.upload_bvh(engine.object_bvh([ctx.object(i) for i in range(ctx.info()["num_objects"])]))
    strat = {}
    for name, code in (("tiled", abi.RKF_STRATEGY_TILED), ("bvh", abi.RKF_STRATEGY_BVH)):
        ps = scenes.march_params(spec)
        ps.strategy = code
        ms = time_view(ctx, cam, ps, args.width, args.height, stream, 5)
        strat[name] = {"mrays": n / ms / 1e3, "ms": ms}
    out["strategies"] = strat
    for name in ("f32", "u8"):
        c2 = Context(pool_capacity=ctx.info()["pool_bricks_used"] + 4096, precision=name, keep_reference_pool=False)
        try:
            c2.voxelize(prims, scenes.voxelize_params(spec, prims))
            ms = time_view(c2, cam, p, args.width, args.height, stream, 5)
            prec[name] = {"mrays": n / ms / 1e3, "ms": ms}
        finally:
            c2.close()
    out["precision_views"] = prec
    out["note"] = "CUDA-event means without the L2 flush of the headline steps"
    return out


def _headline_summary(batching, serving):
    """The metric's comparison in one place: the batched launch and the
    serving loop (at each offered rate) against plain per-request launches
    of the same work, with the loop's p50/p99 latency."""
    if batching is None and serving is None:
        return None
    out = {}
    if batching is not None:
        out["batched"] = {"value": batching["batched"]["value"], "unit": "Mrays/s",
                          "vs_plain": batching["vs_plain"],
                          "vs_b200_per_request": batching["batched"]["value"] / batching["b200_per_request"]["value"],
                          "plain_per_request": batching["plain_per_request"]["value"]}
    if serving is not None:
        out["served"] = [{"rate_hz": r["rate_hz"], "value": r["served"]["value"], "unit": "Mrays/s",
                          "p50_ms": r["served"]["latency_ms"]["p50"], "p99_ms": r["served"]["latency_ms"]["p99"],
                          "vs_plain": r.get("vs_plain")} for r in serving["by_rate"]]
        if "plain_per_request" in serving:
            out["served_plain_per_request"] = serving["plain_per_request"]["value"]
    return out


def run_b200(args, world, rank, local, dist):
    from rkifield_b200 import cudart
    from rkifield_b200.engine import Context, gbuffer_host
    spec = spec_of(args.scene)
    w, h = args.width, args.height
    n = w * h
    cudart.set_device(local)
    cap = args.pool_bricks or (LARGE_POOL if args.scene == "large" else 65_536)
    if args.no_reference_pool:
        args.no_plain = True
    ctx = Context(device=local, pool_capacity=cap, keep_reference_pool=not args.no_reference_pool)
    prims = scenes.make_prims(spec)
    vp = scenes.voxelize_params(spec, prims)
    t0 = time.perf_counter()
    ctx.voxelize(prims, vp)
    build_s = time.perf_counter() - t0
    info = ctx.info()
    cam = camera_for(spec, w, h, rank)
    p = scenes.march_params(spec)
    stream = cudart.Stream()
    g = cudart.device_gbuffer(n)
    gp = cudart.gbuffer_ptrs(g)
    flush = cudart.DeviceArray(256 << 20, np.uint8)
    # set-up, untimed: the autotuner picks the launch tuning for this view and
    # stores it in the context, as a renderer would do once
    import ctypes as C
    vw = (abi.rkf_view * 1)()
    vw[0].camera = cam
    vw[0].width, vw[0].height = w, h
    for k, a in g.items():
        setattr(vw[0].out, k, a.ptr)
    vw[0].out.mem = abi.RKF_MEM_DEVICE
    tu = abi.rkf_batch_tuning()
    t0 = time.perf_counter()
    if args.tuning:
        tu = abi.rkf_batch_tuning(*[int(x) for x in args.tuning.split(",")])
        ctx.set_tuning(tu)
    else:
        abi.check(ctx.lib.rkf_autotune(ctx.h, vw, 1, None, 0, C.byref(p), C.byref(tu)), "autotune")
    tuning = {k: getattr(tu, k) for k, _ in abi.rkf_batch_tuning._fields_}
    tuning["tune_s"] = time.perf_counter() - t0
    tuning["source"] = "--tuning" if args.tuning else "rkf_autotune"

    def launch_stats(cap: int):
        n_launch, n_timed = C.c_uint64(0), C.c_uint32(0)
        kms = (C.c_float * max(cap, 1))()
        abi.check(ctx.lib.rkf_testing_launch_stats(ctx.h, C.byref(n_launch), kms, cap, C.byref(n_timed)),
                  "launch stats")
        return int(n_launch.value), [float(kms[i]) for i in range(min(cap, n_timed.value))]

    def timed(plain: bool, steps: int, warmup: int):
        """Step times (events around the whole call: tile order + march), the
        march kernel's own times (events around its launch alone), the
        library's kernel launches in the timed region and the wall time."""
        for _ in range(warmup):
            ctx.march_async(cam, p, w, h, gp, stream.ptr, plain=plain)
        stream.synchronize()
        ev = [(cudart.Event(), cudart.Event()) for _ in range(steps)]
        barrier(dist)
        cudart.synchronize()
        abi.check(ctx.lib.rkf_testing_march_timing(ctx.h, 1), "march timing")
        launches0, _ = launch_stats(0)
        t_wall = time.perf_counter()
        for a, b in ev:
            flush.memset(1, stream)
            a.record(stream)
            ctx.march_async(cam, p, w, h, gp, stream.ptr, plain=plain)
            b.record(stream)
        stream.synchronize()
        cudart.synchronize()
        barrier(dist)
        wall = time.perf_counter() - t_wall
        launches1, kms = launch_stats(steps)
        abi.check(ctx.lib.rkf_testing_march_timing(ctx.h, 0), "march timing")
        ms = [a.elapsed_ms(b) for a, b in ev]
        return ms, wall, kms, launches1 - launches0

    # e2e: public host-buffer call; pinned host G-buffer copied back each step
    pin = {k: cudart.PinnedArray(v.size, v.dtype) for k, v in gbuffer_host(n).items()}
    host_out = {k: v.array for k, v in pin.items()}

    clk = ClockSampler(local)
    plain = None
    with clk:
        with clk.window():
            ms, wall, kernel_ms, launches = timed(False, args.steps, args.warmup)
        value = job_mrays(dist, world, n, args.steps, sum(ms) / 1e3)
        lat = {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99)),
               "max": float(np.max(ms))}

        if not args.no_plain:
            psteps = max(3, args.steps // 4)
            with clk.window():
                pms, _, _, _ = timed(True, psteps, 1)
            pval = job_mrays(dist, world, n, psteps, sum(pms) / 1e3)
            plain = {"value": pval, "unit": "Mrays/s", "steps": psteps,
                     "latency_ms": {"p50": float(np.percentile(pms, 50)), "p99": float(np.percentile(pms, 99))},
                     "kernel": "k_march_plain (reference AoS pool, one thread per ray, one launch per view)"}

        for _ in range(args.warmup):
            ctx.march(cam, p, w, h, out=host_out)
        barrier(dist)
        with clk.window():
            t0 = time.perf_counter()
            for _ in range(args.steps):
                ctx.march(cam, p, w, h, out=host_out)
            e2e_s = time.perf_counter() - t0
        e2e_val = job_mrays(dist, world, n, args.steps, e2e_s)
    d2h = sum(v.nbytes for v in host_out.values())
    h2d = 144 + 32  # camera uniforms + march parameters

    extras = None
    if args.extras and rank == 0:
        extras = run_extras(args, spec, prims, p, ctx, stream)
    batching = None
    if args.cb_views > 0:
        batching = run_batching(ctx, spec, prims, p, args, stream)
    serving = None
    if args.cs_requests > 0 and rank == 0:
        warm_serving(local)
        # the offered rate, faster ones, and one that saturates the loop
        # (throughput at capacity instead of the offered load)
        rates = [args.cs_rate] + [float(x) for x in args.cs_rates.split(",") if x.strip()]
        if args.cs_sat_rate > 0:
            rates.append(args.cs_sat_rate)
        serving = run_serving(args, spec, prims, p, local, rates)

    out = None
    if rank == 0:
        hits = int((host_out["flags"] & 1).sum())
        roof = None
        cpu = None
        if not (args.no_sectors and args.no_cpu):
            from oracle import binding as oracle
            sc = oracle_scene_from_ctx(ctx, oracle)
            threads = os.cpu_count() or 1
            if not args.no_sectors:
                st = sector_stats(oracle, sc, cam, p, w, h, sample_rows(h, args.sector_rows), threads)
                bytes_per_ray = 24.0 + 32.0 * st["sectors"] / st["rays"]
                bytes_launch = bytes_per_ray * n
                # the march kernel's own launches (the tile-order kernels
                # before it in each step are not part of its roofline)
                mean_s = float(np.mean(kernel_ms if kernel_ms else ms)) / 1e3
                peaks = {}
                pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
                if os.path.exists(pk):
                    peaks = json.load(open(pk))
                peak = peaks.get("hbm_gbs", 6650.0)
                achieved = bytes_launch / mean_s / 1e9
                wl = f"{spec.name} {w}x{h}"
                tr = load_traffic(wl)
                roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": tr,
                        "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback",
                        "algorithmic_bytes_per_ray": bytes_per_ray,
                        "sectors_per_ray": st["sectors"] / st["rays"],
                        "index_sectors_per_ray": st["index_sectors"] / st["rays"],
                        "dist_sectors_per_ray": st["dist_sectors"] / st["rays"],
                        "steps_per_ray": st["steps"] / st["rays"],
                        "sample_rows": args.sector_rows,
                        "kernel_ms": mean_s * 1e3,
                        "kernel_timing": ("CUDA events around the march kernel's launch alone"
                                          if kernel_ms else "CUDA events around the step")}
            if not args.no_cpu:
                rows = sample_rows(h, args.cpu_rows)
                rate, nr, dt = cpu_march_rate(oracle, sc, cam, p, w, h, rows, threads)
                rows1 = sample_rows(h, 2)
                rate1, nr1, dt1 = cpu_march_rate(oracle, sc, cam, p, w, h, rows1, 1)
                cpu = {"value": rate, "unit": "Mrays/s", "cores": threads, "kind": "port",
                       "sample": f"{len(rows)} rows x {w} px ({nr} rays) of the same view, {dt:.1f} s",
                       "single_core": {"value": rate1, "unit": "Mrays/s", "cores": 1,
                                       "sample": f"{len(rows1)} rows x {w} px ({nr1} rays), {dt1:.1f} s"}}
        out = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(ms)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f16 distances)",
            "data": "synthetic (seeded primitives voxelized on the device)",
            "config": {"workload": f"{spec.name} {w}x{h} primary view", "rays_per_step": n,
                       "bricks": info["pool_bricks_used"], "leaf_blocks": info["leaf_blocks"],
                       "build_s": build_s, "hit_fraction": hits / n,
                       "l2": "256 MiB flush between steps, outside the timed events",
                       "tuning": tuning, "parallelism": f"replicas x{world}"},
            "latency_ms": lat,
            "plain": plain,
            "vs_plain": (value / plain["value"]) if plain else None,
            "e2e": {"value": e2e_val, "unit": "Mrays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof,
            "extras": extras,
            "batching": batching,
            "serving": serving,
            "served_batched": _headline_summary(batching, serving),
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "gpu_launches_note": "kernels the library launched in the timed region (march + tile order), "
                                 "counted by the context",
            "wall_s_timed_region": wall,
        }
        print(json.dumps(out), flush=True)
    ctx.close()


def main():
    args = parse()
    world, rank, local, dist = dist_setup()
    try:
        if args.report == "precision":
            if rank == 0:
                if args.scene == "large" and "--scene" in sys.argv:
                    run_precision_report_large(args)
                else:
                    run_precision_report(args)
        elif args.impl == "reference":
            run_reference(args, world, rank, dist)
        else:
            run_b200(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
