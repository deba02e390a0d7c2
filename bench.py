"""Benchmark of the sparse-field level-set hot path (Surface<D,L>::update + Polys) on B200.

Default workload (--config c2): Surface<3,3> float32, 512^3 isogrid with 16^3 partitions,
seeded at the origin and expanded to radius ~100 with 100 untimed steps of speed -1, then timed
steps of delta = -0.2*curv(pos) + 0.1*h(pos, 1234) (h = hashed uniform [-1,1) noise), with
Polys::notify every step and Polys::march every 10th step. A "step" is one Surface::update plus
that repolygonisation. Metric: narrow-band node-updates/s (band size at each step's start).

Config "ray" measures the raycasting row instead: Surface::ray, 2^20 rays per step at the c2
surface (metric rays/s).

Other configs: c1 (Surface<3,2> 64^3, 8^3 partitions, speed -0.5), c3 (4096 Surface<2,2>, grid
edges log-uniform 128..1024, 16^2 partitions, constant speeds U[-0.8,-0.2], marching squares
each step) and c4 (256 Surface<3,2>, edges from {32,48,64,96,128}, 8^3 partitions, speed
-0.3*curv + U[-0.6,0.3], marching cubes at the end), both run as one batch (all surfaces in the
same launches) and also, on a subset, one surface per launch sequence (the plain path).

Arms:
  default           the device engine (libfelt_gpu.so) through its C ABI.
  --impl reference  the reference algorithm's CPU implementation (the oracle port, compiled
                    from oracle/), on the same workload and metric, bounded sample.

Prints ONE JSON line on rank 0. Multi-GPU (torchrun): a single surface does not shard, so for
c1/c2 every rank advances its own replica; for the batched configs every rank advances its own
shard of independent surfaces (same distribution, rank-seeded). No collective touches the data
path; value = all ranks' node-updates / the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c1": dict(kind="single", D=3, L=2, size=(64, 64, 64), part=(8, 8, 8), expand=0,
               speed=dict(c=-0.5), march_every=0, march_end=True, steps=50,
               workload="Surface<3,2> 64^3 / 8^3 partitions, seed at origin, speed -0.5, "
                        "marching cubes at the end"),
    "c2": dict(kind="single", D=3, L=3, size=(512, 512, 512), part=(16, 16, 16), expand=100,
               speed=dict(a=-0.2, n=0.1, seed=1234), march_every=10, march_end=False,
               steps=40,
               workload="Surface<3,3> 512^3 / 16^3 partitions, r~100, speed -0.2*curv + "
                        "0.1*hash_noise, repolygonise every 10 steps"),
    "c3": dict(kind="batch", D=2, L=2, n=4096, part=(16, 16), march_every=1, march_end=False,
               steps=100, plain_subset=16, cpu_subset=16, cpu_steps=100,
               workload="4096 x Surface<2,2>, edges log-uniform 128..1024, 16^2 partitions, "
                        "constant speed U[-0.8,-0.2] per surface, marching squares every step"),
    "c4": dict(kind="batch", D=3, L=2, n=256, part=(8, 8, 8), march_every=0, march_end=True,
               steps=100, plain_subset=16, cpu_subset=4, cpu_steps=50,
               workload="256 x Surface<3,2>, edges from {32,48,64,96,128}, 8^3 partitions, "
                        "speed -0.3*curv + U[-0.6,0.3], marching cubes at the end"),
    "c5": dict(kind="serve", D=3, L=2, part=(8, 8, 8), lambdas=(100, 300, 1000, 3000, 10000),
               max_requests=3000, max_seconds=2.0, budget=150e9, workers=4, plain_subset=24,
               cpu_subset=200,
               workload="served requests, Poisson arrivals at 100..10k/s: Surface<3,2>, edge "
                        "log-uniform 32..256, 8^3 partitions, speed constant U[-0.6,-0.1] | "
                        "-0.3*curv-0.2 | 0.2*hash_noise-0.2, 1..64 steps, polygonise p=0.5, "
                        "admission by a 150 GB brick-pool budget"),
    "local": dict(kind="local", D=3, L=2, size=(256, 256, 256), part=(8, 8, 8), expand=30,
                  box=48, centre=(30, 0, 0), speeds=(-0.2, 0.2), steps=200, cpu_steps=5000,
                  workload="Surface::update(lo, hi, fn) on Surface<3,2> 256^3 / 8^3 partitions, "
                           "r~30 (30 steps of speed -1): each edit a 48^3 box on the surface "
                           "(centre (30,0,0)), constant speed alternating -0.2 / +0.2"),
    "ray": dict(kind="ray", D=3, L=3, size=(512, 512, 512), part=(16, 16, 16), expand=100,
                rays=1 << 20, steps=20, cpu_min_seconds=10.0,
                workload="Surface::ray on Surface<3,3> 512^3 / 16^3 partitions, r~100 (100 "
                         "steps of speed -1): 2^20 rays per step from uniform points on a "
                         "radius-240 sphere, aimed at uniform points within radius 150 of the "
                         "centre"),
}

# Algorithmic bytes per work unit of the kernels whose roofline is reported:
#  k_dist1: per band node of the layer: 2 B list index + 4 B phi read + 4 B delta write.
#  k_dist2: per band node: 2 B list index + 4 B delta read + 4 B phi write.
#  k_delta_*: per zero-layer node: 2 B index + 4 B phi + 4 B delta write.
#  k_flush_*: per leaf edit: 2 B status entry + 1 B to-layer + 2 B lookup read + 2 B list
#             write + 2 B lookup write + 4 B swap-in (moved entry and its lookup).
#  k_polys_march: per cell: 2 B leaf index + 4 B phi (corners are neighbours' phi).
#  k_ray: per ray: origin and direction in, hit out (3 x 12 B in 3D); the nodes it samples
#         are reads of the resident isogrid and are not counted.
UNIT_BYTES = {"k_dist1": (0, 10), "k_dist2": (0, 10), "k_delta_builtin": (1, 10),
              "k_delta_smem": (1, 10), "k_flush_smem": (2, 13), "k_flush_leaf": (2, 13),
              "k_polys_march": (3, 6)}


def batch_surfaces(name, cfg, shard=0):
    """Seeded synthetic surfaces of a batched config: sizes, seed centres, speeds. Under torchrun
    each rank advances its own shard of independent surfaces (shard = rank; shard 0 is the
    single-GPU workload)."""
    import numpy as np
    rng = np.random.default_rng(0x5EED0000 + int(name[1:]) + (shard << 16))
    L, D = cfg["L"], cfg["D"]
    sizes, centres, speeds = [], [], []
    for _ in range(cfg["n"]):
        if name == "c3":
            e = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
            speed = dict(c=float(rng.uniform(-0.8, -0.2)))
        else:
            e = int(rng.choice([32, 48, 64, 96, 128]))
            speed = dict(a=-0.3, c=float(rng.uniform(-0.6, 0.3)))
        size = (e,) * D
        lo, hi = -e // 2 + L + 1, e // 2 - L - 2
        c = tuple(int(rng.integers(lo, hi + 1)) for _ in range(D))
        sizes.append(size)
        centres.append(c)
        speeds.append(speed)
    return sizes, centres, speeds


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu, self.proc, self.lines, self.thread = gpu_index, None, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def combine_ranks(dist, t_ms, wall_s, node_updates, device):
    """Job totals over ranks: the slowest rank's device and wall time, all ranks' node updates."""
    import torch
    mx = torch.tensor([t_ms, wall_s], dtype=torch.float64, device=device)
    sm = torch.tensor([float(node_updates)], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(mx[1]), float(sm[0])


# ---------------------------------------------------------------------------------------------
# Device workloads
# ---------------------------------------------------------------------------------------------

class SingleWork:
    """One Surface (+ Polys) through the C ABI."""

    def __init__(self, fb, cfg, brick_capacity=0):
        self.fb, self.cfg = fb, cfg
        self.s = fb.Surface(cfg["size"], cfg["part"], cfg["L"], brick_capacity=brick_capacity)
        self.p = fb.Polys(self.s)
        self.s.seed((0,) * cfg["D"])
        for _ in range(cfg["expand"]):
            self.s.update(c=-1.0)
        self._pinned()
        # a full polygonisation and readback at setup, so that their buffers exist before timing
        self.p.invalidate()
        self.p.march()
        self.fetch_geometry()

    def step(self, i, last=False):
        c = self.cfg
        self.s.update(**c["speed"])
        self.p.notify()
        if (c["march_every"] and (i + 1) % c["march_every"] == 0) or (last and c["march_end"]):
            self.p.march()
            return True
        return False

    def node_updates(self):
        return self.s.node_updates()

    def stream(self):
        return self.s.stream()

    def work_units(self):
        return self.s.work_units()

    def fetch_geometry(self):
        """D2H of the polygons of the partitions re-marched last (what a viewer would read),
        in one gather call, into pinned host buffers kept between steps."""
        vtx, spx, _ = self.p.gather(self.p.changes(), *self._pinned())
        return vtx.nbytes + spx.nbytes

    def _pinned(self, vfloats=16 << 20, sints=24 << 20):
        """Pinned destination arrays (grown by the gather's own fallback if ever too small)."""
        if getattr(self, "_pv", None) is None:
            import torch
            self._pv = torch.empty(vfloats, dtype=torch.float32, pin_memory=True).numpy()
            self._ps = torch.empty(sints, dtype=torch.int32, pin_memory=True).numpy().view(
                "uint32")
        return self._pv, self._ps


class BatchWork:
    """All surfaces of a batched config in one batch."""

    def __init__(self, fb, cfg, name, shard=0):
        self.fb, self.cfg = fb, cfg
        sizes, centres, speeds = batch_surfaces(name, cfg, shard)
        self.b = fb.Batch(sizes, cfg["part"], cfg["L"])
        self.b.seed(centres)
        self.speeds = self.b.speed_array(speeds)  # converted once; the speeds are fixed
        # a full polygonisation at setup, so that its buffers exist before timing
        self.b.polys_invalidate()
        self.b.polys_march()
        self.b.polys_totals()
        self.surface0 = None

    def step(self, i, last=False):
        c = self.cfg
        self.b.update(self.speeds)
        self.b.polys_notify()
        if (c["march_every"] and (i + 1) % c["march_every"] == 0) or (last and c["march_end"]):
            self.b.polys_march()
            return True
        return False

    def node_updates(self):
        return self.b.node_updates()

    def stream(self):
        return self.b.stream()

    def work_units(self):
        return self.b.work_units()

    def fetch_geometry(self):
        """Polygon counts of the batch (a viewer of many small surfaces reads totals)."""
        self.b.polys_totals()
        return 16


class PlainSubset:
    """The plain path on the first k surfaces of a batched config: one Surface each, advanced
    one surface at a time (every update its own launch sequence)."""

    def __init__(self, fb, cfg, name, k):
        sizes, centres, speeds = batch_surfaces(name, cfg)
        self.cfg = cfg
        self.items = []
        for sz, c, sp in list(zip(sizes, centres, speeds))[:k]:
            s = fb.Surface(sz, cfg["part"], cfg["L"])
            s.seed(c)
            self.items.append((s, fb.Polys(s), sp))

    def step(self, i, last=False):
        c = self.cfg
        keep = []
        for s, p, sp in self.items:
            try:
                s.update(**sp)
            except Exception:  # stopped: its convergence loop did not terminate
                self.done += s.node_updates()
                continue
            p.notify()
            if (c["march_every"] and (i + 1) % c["march_every"] == 0) or (last and c["march_end"]):
                p.march()
            keep.append((s, p, sp))
        self.items = keep

    done = 0

    def node_updates(self):
        return self.done + sum(s.node_updates() for s, _, _ in self.items)


def time_steps(torch, work, stream, steps, warm, flush, start=0, profile=False):
    """Times `steps` steps two ways over the same work: device time (CUDA events on the work's
    stream around the update/polygonisation launches) and end-to-end wall time through the C
    ABI (the host-side speed structs going in, the step's result coming out: the node-update
    counter every step and, after a march, the re-marched polygons). L2 is flushed (256 MB
    write, > 126 MB L2) before each step, outside both timed intervals. With profile, the timed
    steps run between cudaProfilerStart and cudaProfilerStop (for ncu --profile-from-start off).
    """
    for i in range(warm):
        work.step(start + i)
    torch.cuda.synchronize()
    if profile:
        u0 = work.work_units()
        torch.cuda.profiler.start()
    nu0 = work.node_updates()
    total, wall, d2h = 0.0, 0.0, 0
    for i in range(steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        marched = work.step(start + warm + i, last=(i == steps - 1))
        b.record(stream)
        if marched:
            d2h += work.fetch_geometry()
        work.node_updates()
        d2h += 8
        wall += time.perf_counter() - t0
        b.synchronize()
        total += a.elapsed_time(b)
    torch.cuda.synchronize()
    if profile:
        torch.cuda.profiler.stop()
        u1 = work.work_units()
        print("profiled region work units (dist, zero, flush, march): "
              + json.dumps([b - a for a, b in zip(u0, u1)]), file=sys.stderr, flush=True)
    return total, wall, work.node_updates() - nu0, d2h


# ---------------------------------------------------------------------------------------------
# CPU (oracle port)
# ---------------------------------------------------------------------------------------------

def cpu_threads():
    """Sets the oracle's parallel loops (those the reference runs with OpenMP) to every host
    core; returns the thread count."""
    from oracle import oracle as O
    return O.set_threads(os.cpu_count() or 1)


def cpu_single(cfg, steps, warm=3):
    from oracle import oracle as O
    s = O.Surface(cfg["size"], cfg["part"], cfg["L"])
    p = O.Polys(s)
    s.seed((0,) * cfg["D"])
    if cfg["expand"]:
        s.run_steps(cfg["expand"], c=-1.0)
    for _ in range(warm):
        s.update(**cfg["speed"])
        p.notify()
    nu, secs = 0.0, 0.0
    for i in range(steps):
        nu += s.band_size()
        t0 = time.perf_counter()
        s.update(**cfg["speed"])
        p.notify()
        if (cfg["march_every"] and (i + 1) % cfg["march_every"] == 0) or (
                i == steps - 1 and cfg["march_end"]):
            p.march()
        secs += time.perf_counter() - t0
    return nu / secs, nu, secs


def cpu_batch(name, cfg, steps, k):
    from oracle import oracle as O
    sizes, centres, speeds = batch_surfaces(name, cfg)
    items = []
    for sz, c, sp in list(zip(sizes, centres, speeds))[:k]:
        s = O.Surface(sz, cfg["part"], cfg["L"])
        s.seed(c)
        items.append((s, O.Polys(s), sp))
    nu, secs = 0.0, 0.0
    for i in range(steps):
        keep = []
        for s, p, sp in items:
            band = s.band_size()
            t0 = time.perf_counter()
            try:
                s.update(**sp)
            except O.OracleError:  # the reference's loop would not terminate: drop it
                secs += time.perf_counter() - t0
                continue
            p.notify()
            if (cfg["march_every"] and (i + 1) % cfg["march_every"] == 0) or (
                    i == steps - 1 and cfg["march_end"]):
                p.march()
            secs += time.perf_counter() - t0
            nu += band
            keep.append((s, p, sp))
        items = keep
    return nu / secs, nu, secs


def cpu_baseline(name, cfg, steps):
    threads = cpu_threads()
    if cfg["kind"] == "single":
        rate, nu, secs = cpu_single(cfg, steps)
        sample = f"{steps} timed steps after the same setup"
    else:
        k = cfg["cpu_subset"]
        rate, nu, secs = cpu_batch(name, cfg, steps, k)
        sample = f"first {k} surfaces of the workload, {steps} steps each, one after another"
    out = {"value": rate, "unit": "node-updates/s", "cores": threads, "kind": "port",
           "sample": f"{sample} ({nu:.3g} node-updates in {secs:.2f} s; the reference's "
                     f"parallel loops on {threads} threads)"}
    # a step of a single-surface config is the whole workload's step; a batch config's sample
    # is a subset of its surfaces, so its time is not a step of the workload
    step_ms = secs * 1e3 / steps if cfg["kind"] == "single" and steps else None
    return out, step_ms


def run_reference(args, name, cfg):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    metric, unit = "narrow-band node-updates/s", "node-updates/s"
    step_ms = None
    if cfg["kind"] == "serve":
        steps = None
        base = serve_cpu(cfg, cfg["cpu_subset"])
    elif cfg["kind"] == "ray":
        steps = 1
        base = cpu_rays(cfg)
        metric, unit = "rays/s", "rays/s"
    elif cfg["kind"] == "local":
        steps = cfg["cpu_steps"]
        base = cpu_local(cfg)
        metric, unit = "local edits/s", "edits/s"
    else:
        steps = args.steps or cfg["steps"]
        steps = min(steps, 20 if cfg["kind"] == "single" else 10)
        base, step_ms = cpu_baseline(name, cfg, steps)
    line = {
        "impl": "reference", "metric": metric, "value": base["value"],
        "unit": unit, "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "name": name},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# Device arm
# ---------------------------------------------------------------------------------------------

def roofline(fb, work, cfg, stream_steps):
    units0 = work.work_units()
    fb.profile_reset()
    fb.profile_enable(True)
    for i in range(stream_steps):
        work.step(10_000 + i, last=(i == stream_steps - 1))
    import torch
    torch.cuda.synchronize()
    fb.profile_enable(False)
    prof = fb.profile_read()
    units1 = work.work_units()
    tot = sum(v[0] for v in prof.values())
    ranked = sorted(prof.items(), key=lambda kv: -kv[1][0])
    hbm, peak_kind = load_peaks()
    out = {"bound": "hbm", "peak": hbm, "unit": "GB/s", "peak_kind": peak_kind,
           "kernel_ms_per_step": tot / stream_steps,
           "top_kernels": [[k, round(v[0] / tot, 4), v[1]] for k, v in ranked[:10]]}
    dom = next((k for k, _ in ranked if k in UNIT_BYTES), None)
    if dom and any(units1[i] - units0[i] for i in range(4)):
        ms, nl = prof[dom]
        ui, per = UNIT_BYTES[dom]
        units = units1[ui] - units0[ui]
        bpl = per * units / nl
        achieved = bpl / (ms / nl * 1e-3) / 1e9
        out.update({"kernel": dom, "achieved": achieved, "frac": achieved / hbm,
                    "traffic": None, "bytes_per_launch": bpl, "avg_launch_us": 1e3 * ms / nl,
                    "share_of_step_kernel_time": ms / tot})
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            try:
                t = json.load(open(tf)).get(dom)
                if t:
                    out["traffic"] = t["bytes_per_unit"] * units / nl
            except Exception:
                pass
    return out


def ray_inputs(cfg, n, seed):
    """Seeded rays of the ray config: origins uniform on a radius-240 sphere, each aimed at a
    point uniform in the radius-150 ball around the centre; float32, unit directions."""
    import numpy as np
    rng = np.random.default_rng(seed)
    D = cfg["D"]
    u = rng.normal(size=(n, D))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    o = u * 240.0
    v = rng.normal(size=(n, D))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    tgt = v * 150.0 * rng.random((n, 1)) ** (1.0 / D)
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o.astype(np.float32), d.astype(np.float32)


def cpu_rays(cfg, seed=0):
    """The oracle's Surface::ray over the config's rays on every host core, passes over the
    same 2^20 rays until cpu_min_seconds of casting have elapsed."""
    import numpy as np
    from oracle import oracle as O
    threads = cpu_threads()
    s = O.Surface(cfg["size"], cfg["part"], cfg["L"])
    s.seed((0,) * cfg["D"])
    s.run_steps(cfg["expand"], c=-1.0)
    o, d = ray_inputs(cfg, cfg["rays"], seed)
    n, secs, passes = 0, 0.0, 0
    while secs < cfg["cpu_min_seconds"] and passes < 20:
        t0 = time.perf_counter()
        s.rays(o, d)
        secs += time.perf_counter() - t0
        n += o.shape[0]
        passes += 1
    return {"value": n / secs, "unit": "rays/s", "cores": threads, "kind": "port",
            "sample": f"{passes} pass(es) over the {o.shape[0]} rays of the workload on the "
                      f"same surface ({n} rays in {secs:.2f} s, rays spread over {threads} "
                      f"threads)"}


def run_ray(args, name, cfg):
    """Surface::ray throughput: value = rays/s of the device kernel with rays resident in HBM;
    e2e = rays/s through fg_ray with pinned host arrays (copies in, hits out)."""
    import ctypes as C
    import numpy as np
    import torch
    import felt_b200 as fb
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    steps = args.steps or cfg["steps"]
    s = fb.Surface(cfg["size"], cfg["part"], cfg["L"], brick_capacity=args.brick_capacity)
    s.seed((0,) * cfg["D"])
    for _ in range(cfg["expand"]):
        s.update(c=-1.0)
    n = cfg["rays"]
    o, d = ray_inputs(cfg, n, seed=rank)
    to, td = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    th = torch.empty_like(to)
    ho = torch.from_numpy(o).pin_memory()
    hd = torch.from_numpy(d).pin_memory()
    hh = torch.empty_like(ho).pin_memory()
    stream = torch.cuda.ExternalStream(s.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    lib = fb.lib()

    def cast_device():
        s.rays_device(to.data_ptr(), td.data_ptr(), n, th.data_ptr())

    def cast_host():
        fb._chk(lib.fg_ray(s._h, C.c_void_p(ho.data_ptr()), C.c_void_p(hd.data_ptr()),
                           C.c_size_t(n), C.c_void_p(hh.data_ptr())))

    for _ in range(args.warmup):
        cast_device()
        cast_host()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = fb.launch_count()
    total = 0.0
    step_ms = []
    for i in range(steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cast_device()
        b.record(stream)
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
        total += step_ms[-1]
    wall = 0.0
    for i in range(steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cast_host()
        wall += time.perf_counter() - t0
    launches = fb.launch_count() - l0
    clk = clocks.stop()
    torch.cuda.synchronize()
    hits = float(np.mean(np.any(th.cpu().numpy() != np.float32(np.finfo(np.float32).max),
                                axis=1)))
    same = bool(torch.equal(th.cpu(), hh))
    if pg:
        t_ms, wall, _ = combine_ranks(pg, total, wall, 0.0, "cuda")
        total = t_ms
    value = ws * n * steps / (total / 1e3)
    e2e = {"value": ws * n * steps / wall, "unit": "rays/s",
           "h2d_bytes_per_step": 2 * o.nbytes, "d2h_bytes_per_step": o.nbytes,
           "how": "fg_ray with pinned host arrays, wall clock, copies inside"}
    roof = None
    cpu = None
    if rank == 0:
        fb.profile_reset()
        fb.profile_enable(True)
        for _ in range(3):
            cast_device()
        torch.cuda.synchronize()
        fb.profile_enable(False)
        prof = fb.profile_read()
        # one cast = k_ray_ranges, k_ray_walk, k_ray_march, k_ray_find, k_ray_conv (plus
        # k_ray_find and k_ray_conv again per resumed round, rare); the roofline covers them all
        ms = sum(v[0] for k, v in prof.items() if k.startswith("k_ray"))
        calls = 3
        hbm, peak_kind = load_peaks()
        per = 3 * 4 * cfg["D"]
        achieved = per * n / (ms / calls * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "k_ray_walk+march+conv", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "peak_kind": peak_kind, "frac": achieved / hbm,
                "traffic": None, "bytes_per_launch": per * n, "avg_launch_us": 1e3 * ms / calls,
                "kernels": {k: {"ms_per_cast": v[0] / calls, "launches": v[1]}
                            for k, v in prof.items()}}
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            t = json.load(open(tf)).get("k_ray_walk+march+conv")
            if t:
                roof["traffic"] = t["bytes_per_unit"] * n
        if ws == 1 and not args.no_cpu:
            cpu = cpu_rays(cfg)
        config = {"workload": cfg["workload"], "name": name, "rays_per_step": n,
                  "step_ms": [round(x, 2) for x in step_ms],
                  "parallelism": f"replicas{ws}", "hit_fraction": hits,
                  "device_and_host_paths_agree": same,
                  "l2": "flushed between timed steps (256 MB write)"}
        line = {
            "metric": "rays/s", "value": value, "unit": "rays/s", "n_gpus": ws,
            "steps": steps, "warmup": args.warmup, "ms_per_step": total / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config, "roofline": roof, "cpu_baseline": cpu,
            "e2e": e2e, "clocks": clk, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def local_box(cfg):
    h = cfg["box"] // 2
    return ([c - h for c in cfg["centre"]], [c + h for c in cfg["centre"]])


def cpu_local(cfg):
    """The oracle's bounded updates: the same edits on the same surface, one after another, on
    one thread (the oracle starts threads per parallel loop, which costs these small edits more
    than it saves: one thread is its fastest here)."""
    from oracle import oracle as O
    threads = O.set_threads(1)
    s = O.Surface(cfg["size"], cfg["part"], cfg["L"])
    s.seed((0,) * cfg["D"])
    s.run_steps(cfg["expand"], c=-1.0)
    lo, hi = local_box(cfg)
    secs = 0.0
    n = cfg["cpu_steps"]
    for i in range(n):
        t0 = time.perf_counter()
        s.update_bounded(lo, hi, c=cfg["speeds"][i % 2])
        secs += time.perf_counter() - t0
    return {"value": n / secs, "unit": "edits/s", "cores": threads, "kind": "port",
            "sample": f"{n} edits of the workload after the same setup ({secs:.2f} s on "
                      f"{threads} thread, the oracle's fastest setting for edits this small)"}


def run_local(args, name, cfg):
    """Interactive edits: value = bounded updates per second, device-timed; e2e = the same
    through the C ABI with the band size read back after each edit."""
    import torch
    import felt_b200 as fb
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    steps = args.steps or cfg["steps"]
    s = fb.Surface(cfg["size"], cfg["part"], cfg["L"], brick_capacity=args.brick_capacity)
    s.seed((0,) * cfg["D"])
    for _ in range(cfg["expand"]):
        s.update(c=-1.0)
    lo, hi = local_box(cfg)
    sp = cfg["speeds"]
    for i in range(max(args.warmup, 2) * 2):
        s.update_bounded(lo, hi, c=sp[i % 2])
    stream = torch.cuda.ExternalStream(s.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = fb.launch_count()
    total = 0.0
    if args.profile_region:
        torch.cuda.profiler.start()
    for i in range(steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.update_bounded(lo, hi, c=sp[i % 2])
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    if args.profile_region:
        torch.cuda.profiler.stop()
    wall = 0.0
    for i in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.update_bounded(lo, hi, c=sp[i % 2])
        s.band_size()
        wall += time.perf_counter() - t0
    launches = fb.launch_count() - l0
    clk = clocks.stop()
    if pg:
        total, wall, _ = combine_ranks(pg, total, wall, 0.0, "cuda")
    value = ws * steps / (total / 1e3)
    cpu = None
    if rank == 0:
        if ws == 1 and not args.no_cpu:
            cpu = cpu_local(cfg)
        config = {"workload": cfg["workload"], "name": name, "parallelism": f"replicas{ws}",
                  "band_nodes": s.band_size(),
                  "l2": "flushed between timed edits (256 MB write)"}
        line = {
            "metric": "local edits/s", "value": value, "unit": "edits/s", "n_gpus": ws,
            "steps": steps, "warmup": args.warmup, "ms_per_step": total / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config, "roofline": None, "cpu_baseline": cpu,
            "e2e": {"value": ws * steps / wall, "unit": "edits/s", "h2d_bytes_per_step": 44,
                    "d2h_bytes_per_step": 8,
                    "how": "fg_update_bounded then the band size read back, wall clock"},
            "clocks": clk, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def serve_requests(cfg, lam, shard=0):
    """Seeded Poisson request stream at rate lam: (arrival offset s, Request) pairs."""
    import numpy as np
    from felt_b200.serving import Request
    rng = np.random.default_rng(0x5EED0005 + int(lam) + (shard << 20))
    L = cfg["L"]
    n = int(min(cfg["max_requests"], lam * cfg["max_seconds"]))
    t, out = 0.0, []
    for k in range(n):
        t += float(rng.exponential(1.0 / lam))
        e = int(round(math.exp(rng.uniform(math.log(32), math.log(256)))))
        kind = ("constant", "curvature", "noise")[int(rng.integers(0, 3))]
        if kind == "constant":
            sp = dict(c=float(rng.uniform(-0.6, -0.1)))
        elif kind == "curvature":
            sp = dict(a=-0.3, c=-0.2)
        else:
            sp = dict(n=0.2, seed=int(rng.integers(0, 2**31)), c=-0.2)
        lo, hi = -e // 2 + L + 1, e // 2 - L - 2
        c = tuple(int(rng.integers(lo, hi + 1)) for _ in range(3))
        steps = int(rng.integers(1, 65))
        polys = bool(rng.random() < 0.5)
        out.append((t, Request((e, e, e), c, sp, steps, polys, kind, rid=k)))
    return out


def serve_one_rate(fb, cfg, lam, shard=0):
    """Feeds one rate's stream into a Server in real time; latency and throughput figures."""
    from felt_b200.serving import Server
    stream = serve_requests(cfg, lam, shard)
    srv = Server(layers=cfg["L"], part=cfg["part"], budget_bytes=cfg["budget"],
                 workers=cfg["workers"])
    try:
        t_first = srv.now()
        for off, req in stream:
            due = t_first + off
            while srv.now() < due:
                time.sleep(min(0.0005, max(0.0, due - srv.now())))
            req.arrival = due
            srv.submit(req)
        if not srv.drain(timeout=900):
            raise RuntimeError("serving did not drain")
        res = srv.results()
        t_end = max((r.done for r in res), default=t_first)
        lat = sorted(r.latency for r in res)
        pct = (lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] * 1e3) if lat else (lambda q: None)
        return {"lambda_per_s": lam, "requests": len(stream), "admitted": srv.admitted,
                "rejected": srv.rejected, "stopped": sum(r.stopped for r in res),
                "p50_ms": pct(0.50), "p99_ms": pct(0.99),
                "node_updates_per_s": srv.node_updates / max(t_end - t_first, 1e-9),
                "node_updates": srv.node_updates, "seconds": t_end - t_first}
    finally:
        srv.close()


def serve_plain(fb, cfg, k):
    """The plain path on the first k requests of the 1k/s stream: one Surface (+ Polys) per
    request, one request after another, wall clock."""
    reqs = [r for _, r in serve_requests(cfg, 1000)[:k]]
    nu, secs = 0, 0.0
    for r in reqs:
        t0 = time.perf_counter()
        s = fb.Surface(r.size, cfg["part"], cfg["L"])
        p = fb.Polys(s)
        s.seed(r.centre)
        for _ in range(r.steps):
            s.update(**r.speed)
            p.notify()
        if r.polys:
            p.march()
        n = s.node_updates()
        secs += time.perf_counter() - t0
        nu += n
        del p, s
    return nu / secs, nu, secs


def serve_cpu(cfg, k):
    """The oracle on the first k requests of the 1k/s stream, one after another."""
    from oracle import oracle as O
    threads = cpu_threads()
    reqs = [r for _, r in serve_requests(cfg, 1000)[:k]]
    nu, secs = 0.0, 0.0
    for r in reqs:
        s = O.Surface(r.size, cfg["part"], cfg["L"])
        p = O.Polys(s)
        s.seed(r.centre)
        for _ in range(r.steps):
            band = s.band_size()
            t0 = time.perf_counter()
            try:
                s.update(**r.speed)
            except O.OracleError:
                secs += time.perf_counter() - t0
                break
            p.notify()
            secs += time.perf_counter() - t0
            nu += band
        if r.polys:
            t0 = time.perf_counter()
            p.march()
            secs += time.perf_counter() - t0
    return {"value": nu / secs, "unit": "node-updates/s", "cores": threads, "kind": "port",
            "sample": f"first {k} requests of the 1k/s stream, one after another "
                      f"({nu:.3g} node-updates in {secs:.2f} s; the reference's parallel "
                      f"loops on {threads} threads)"}


def run_serve(args, name, cfg):
    import torch
    import felt_b200 as fb
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    # warm-up: one small wave through every code path
    serve_one_rate(fb, dict(cfg, max_requests=8), 1000, shard=rank)
    clocks = ClockSampler(local)
    clocks.start()
    l0 = fb.launch_count()
    sweep = [serve_one_rate(fb, cfg, lam, shard=rank) for lam in cfg["lambdas"]]
    launches = fb.launch_count() - l0
    clk = clocks.stop()
    best = max(sweep, key=lambda r: r["node_updates_per_s"])
    value = best["node_updates_per_s"]
    if pg:
        secs, _, nu = combine_ranks(pg, best["seconds"], 0.0, best["node_updates"], "cuda")
        value = nu / secs
    extra = {}
    cpu = None
    if rank == 0:
        p_rate, _, _ = serve_plain(fb, cfg, cfg["plain_subset"])
        extra["plain"] = {"value": p_rate, "unit": "node-updates/s",
                          "requests": cfg["plain_subset"],
                          "how": "one Surface per request, requests one after another, wall clock"}
        extra["served_over_plain"] = value / p_rate
        if ws == 1 and not args.no_cpu:
            cpu = serve_cpu(cfg, cfg["cpu_subset"])
    if rank == 0:
        config = {"workload": cfg["workload"], "name": name,
                  "parallelism": f"surface shards x{ws} (independent request streams per rank)",
                  "sweep": sweep, "value_at_lambda": best["lambda_per_s"]}
        config.update(extra)
        line = {
            "metric": "narrow-band node-updates/s", "value": value, "unit": "node-updates/s",
            "n_gpus": ws, "steps": None, "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config, "roofline": None, "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "node-updates/s", "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": None,
                    "how": "wall clock from each request's arrival to its result, through the "
                           "public API"},
            "clocks": clk, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_felt(args, name, cfg):
    import torch
    import felt_b200 as fb

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    steps = args.steps or cfg["steps"]
    work = (SingleWork(fb, cfg, args.brick_capacity) if cfg["kind"] == "single"
            else BatchWork(fb, cfg, name, shard=rank))
    stream = torch.cuda.ExternalStream(work.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = fb.launch_count()
    print(f"launches before the timed region: {l0}", file=sys.stderr, flush=True)
    t_ms, wall_s, nu, d2h = time_steps(torch, work, stream, steps, args.warmup, flush,
                                       profile=args.profile_region)
    launches = fb.launch_count() - l0
    clk = clocks.stop()
    if pg:
        t_ms, wall_s, nu = combine_ranks(pg, t_ms, wall_s, nu, "cuda")
    value = nu / (t_ms / 1e3)
    import ctypes as C
    e2e = {"value": nu / wall_s, "unit": "node-updates/s",
           "h2d_bytes_per_step": C.sizeof(fb.Speed) * (cfg.get("n") or 1),
           "d2h_bytes_per_step": d2h // steps}

    extra = {}
    roof = None
    if rank == 0:
        roof = roofline(fb, work, cfg, max(cfg["march_every"] or 5, 5))
        if cfg["kind"] == "batch" and not args.no_plain:
            plain = PlainSubset(fb, cfg, name, cfg["plain_subset"])
            ps = torch.cuda.ExternalStream(0)
            p_steps = min(steps, 10)
            t0 = time.perf_counter()
            nu0 = plain.node_updates()
            for i in range(p_steps):
                plain.step(i, last=(i == p_steps - 1))
            torch.cuda.synchronize()
            p_rate = (plain.node_updates() - nu0) / (time.perf_counter() - t0)
            del ps
            extra["plain"] = {"value": p_rate, "unit": "node-updates/s",
                              "surfaces": cfg["plain_subset"], "steps": p_steps,
                              "how": "one Surface per launch sequence, surfaces one after "
                                     "another, wall clock"}
            extra["batched_over_plain"] = value / p_rate
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu, _ = cpu_baseline(name, cfg, args.cpu_steps if cfg["kind"] == "single"
                              else cfg["cpu_steps"])

    if rank == 0:
        par = (f"replicas{ws}" if cfg["kind"] == "single"
               else f"surface shards x{ws} (independent surfaces per rank)")
        config = {"workload": cfg["workload"], "name": name, "parallelism": par,
                  "l2": "flushed between timed steps (256 MB write)", "node_updates": nu}
        config.update(extra)
        line = {
            "metric": "narrow-band node-updates/s", "value": value, "unit": "node-updates/s",
            "n_gpus": ws, "steps": steps, "warmup": args.warmup, "ms_per_step": t_ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config, "roofline": roof, "cpu_baseline": cpu,
            "e2e": e2e, "clocks": clk, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0, help="timed steps (default per config)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="felt", choices=["felt", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--brick-capacity", type=int, default=0,
                    help="brick pool capacity of single-surface configs (0 = automatic)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, args.config, cfg)
    elif cfg["kind"] == "serve":
        run_serve(args, args.config, cfg)
    elif cfg["kind"] == "ray":
        run_ray(args, args.config, cfg)
    elif cfg["kind"] == "local":
        run_local(args, args.config, cfg)
    else:
        run_felt(args, args.config, cfg)


if __name__ == "__main__":
    main()
