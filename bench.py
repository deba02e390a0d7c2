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
               max_requests=3000, max_seconds=2.0, budget=150e9, slots=512,
               max_size=(256, 256, 256), plain_subset=24, cpu_subset=200,
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

# Algorithmic bytes: 16 B per narrow-band node-update (a 4 B list index read, a 4 B value read,
# a 4 B value write and 4 B of per-node auxiliary traffic: the delta of a zero-layer node, the
# status or list write of the others; neighbour reads are other nodes' value reads and are not
# counted twice). A kernel's launch is credited 16 B per work unit it processes: band nodes for
# the distance passes, zero-layer nodes for the speed functor and the zero-layer update, leaf
# edits for the status-change flush, cells for the march.
BYTES_PER_NODE_UPDATE = 16
UNIT_OF = {"k_dist1": 0, "k_dist2": 0, "k_delta_builtin": 1, "k_delta_smem": 1,
           "k_zero_apply": 1, "k_flush_smem": 2, "k_flush_leaf": 2, "k_polys_march": 3}


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

# Launch tuning of every surface and batch the bench creates (fg_config: launch_mode,
# autotune), from the command line.
TUNING = {}
# Device time of each step of the last timed run (ms).
STEP_MS = []


class SingleWork:
    """One Surface (+ Polys) through the C ABI."""

    def __init__(self, fb, cfg, brick_capacity=0):
        self.fb, self.cfg = fb, cfg
        # the polygon arena sized for the surface's geometry with the polygoniser's headroom
        # (16x the live vertices: C2 holds up to ~0.7 M), so that no timed march grows it
        self.s = fb.Surface(cfg["size"], cfg["part"], cfg["L"], brick_capacity=brick_capacity,
                            vertex_capacity=1 << 24, **TUNING)
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
        self.s.update(**self.cfg["speed"])
        self.p.notify()
        if march_due(self.cfg, i, last):
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

    def close(self):
        self.p.close()
        self.s.close()

    def tuning(self):
        return self.s.tuning()

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
        # threads per brick from the launch-shape tuner (fg_autotune), as the batched configs ask
        self.b = fb.Batch(sizes, cfg["part"], cfg["L"], **{**TUNING, "autotune": True})
        self.b.seed(centres)
        self.speeds = self.b.speed_array(speeds)  # converted once; the speeds are fixed
        # a full polygonisation at setup, so that its buffers exist before timing
        self.b.polys_invalidate()
        self.b.polys_march()
        self.b.polys_totals()
        self.surface0 = None

    def step(self, i, last=False):
        self.b.update(self.speeds)
        self.b.polys_notify()
        if march_due(self.cfg, i, last):
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

    def close(self):
        self.b.close()

    def tuning(self):
        return self.b.tuning()


class PlainSubset:
    """The plain path on the first k surfaces of a batched config: one Surface each, advanced
    one surface at a time (every update its own launch sequence). step() times each surface's
    update and polygonisation with CUDA events on that surface's stream, so the plain path has
    a device time like the batch's."""

    def __init__(self, fb, cfg, name, k):
        sizes, centres, speeds = batch_surfaces(name, cfg)
        self.cfg = cfg
        self.items = []
        self.done = 0
        for sz, c, sp in list(zip(sizes, centres, speeds))[:k]:
            s = fb.Surface(sz, cfg["part"], cfg["L"], **{**TUNING, "autotune": True})
            s.seed(c)
            self.items.append((s, fb.Polys(s), sp))

    def step(self, i, last=False, torch=None):
        """One step of every surface; returns the device time of the step in ms (summed over
        the surfaces' streams) when torch is given."""
        dev_ms = 0.0
        keep = []
        for s, p, sp in self.items:
            if torch is not None:
                st = torch.cuda.ExternalStream(s.stream())
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(st)
            try:
                s.update(**sp)
            except Exception:  # stopped: its convergence loop did not terminate
                self.done += s.node_updates()
                continue
            p.notify()
            if march_due(self.cfg, i, last):
                p.march()
            if torch is not None:
                b.record(st)
                b.synchronize()
                dev_ms += a.elapsed_time(b)
            keep.append((s, p, sp))
        self.items = keep
        return dev_ms

    def node_updates(self):
        return self.done + sum(s.node_updates() for s, _, _ in self.items)

    def close(self):
        for s, p, _ in self.items:
            p.close()
            s.close()
        self.items = []


def measure_batched(fb, name, steps, warm):
    """The batched workload against the plain path on the same surfaces and steps: every
    surface of the config in one batch (the same launches for all), and its first
    `plain_subset` surfaces one Surface each, one after another. Both are timed two ways over
    the same steps: device time (CUDA events on the launching streams) and wall clock with the
    host calls and synchronisation. The ratios compare like with like."""
    import torch
    cfg = CONFIGS[name]
    work = BatchWork(fb, cfg, name)
    stream = torch.cuda.ExternalStream(work.stream())
    for i in range(warm):
        work.step(i)
    torch.cuda.synchronize()
    nu0 = work.node_updates()
    dev_ms, wall = 0.0, 0.0
    for i in range(steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        work.step(warm + i, last=(i == steps - 1))
        b.record(stream)
        b.synchronize()
        wall += time.perf_counter() - t0
        dev_ms += a.elapsed_time(b)
    nu = work.node_updates() - nu0
    tuning = work.tuning()
    work.close()
    k = cfg["plain_subset"]
    plain = PlainSubset(fb, cfg, name, k)
    for i in range(warm):
        plain.step(i)
    torch.cuda.synchronize()
    pnu0 = plain.node_updates()
    pdev_ms, pwall = 0.0, 0.0
    for i in range(steps):
        t0 = time.perf_counter()
        pdev_ms += plain.step(warm + i, last=(i == steps - 1), torch=torch)
        torch.cuda.synchronize()
        pwall += time.perf_counter() - t0
    pnu = plain.node_updates() - pnu0
    plain.close()
    b_dev, b_wall = nu / (dev_ms * 1e-3), nu / wall
    p_dev, p_wall = pnu / (pdev_ms * 1e-3), pnu / pwall
    return {"workload": cfg["workload"], "name": name, "steps": steps, "warmup": warm,
            "batched": {"surfaces": cfg["n"], "node_updates": nu, "device_per_s": b_dev,
                        "wall_per_s": b_wall, "ms_per_step": dev_ms / steps},
            "plain": {"surfaces": k, "node_updates": pnu, "device_per_s": p_dev,
                      "wall_per_s": p_wall, "ms_per_step": pdev_ms / steps},
            "batched_over_plain_device": b_dev / p_dev,
            "batched_over_plain_wall": b_wall / p_wall,
            "tuning": tuning,
            "how": "node-updates/s of the same steps; batched: all surfaces in one batch; plain: "
                   "the first surfaces as separate Surfaces one after another (every update its "
                   "own launch sequence); device = CUDA events on the launching streams, wall = "
                   "host clock around the calls with synchronisation"}


def measure_served(fb, name, lambdas):
    """The served workload at the given arrival rates, and the plain path on the same request
    mix (one Surface per request, one request after another, seed to result, wall clock)."""
    from felt_b200.serving import Server
    cfg = CONFIGS[name]
    budget = serve_budget(cfg)
    srv = Server(layers=cfg["L"], part=cfg["part"], budget_bytes=budget, slots=cfg["slots"],
                 max_size=cfg["max_size"])
    try:
        serve_one_rate(srv, cfg, 1000,
                       stream=[(t, r) for t, r in serve_requests(cfg, 1000, shard=99)[:16]])
        sweep = [serve_one_rate(srv, cfg, lam) for lam in lambdas]
    finally:
        srv.close()
    p_rate, p_nu, p_secs, p_make = serve_plain(fb, cfg, cfg["plain_subset"])
    best = max(sweep, key=lambda r: r["node_updates_per_s"])
    return {"workload": cfg["workload"], "name": name, "budget_bytes": budget,
            "slots": cfg["slots"], "sweep": sweep, "best_lambda_per_s": best["lambda_per_s"],
            "node_updates_per_s": best["node_updates_per_s"],
            "plain": {"node_updates_per_s": p_rate, "requests": cfg["plain_subset"],
                      "seconds": p_secs, "surface_create_s": p_make,
                      "how": "one Surface per request, requests one after another, wall clock "
                             "from seed to result (construction timed apart)"},
            "served_over_plain": best["node_updates_per_s"] / p_rate,
            "how": "wall clock from each request's scheduled arrival to its result on the "
                   "server's clock; throughput = node updates of the rate's requests / the time "
                   "from its first arrival to its last result"}


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
    per_step = []
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
        per_step.append(a.elapsed_time(b))
        total += per_step[-1]
    torch.cuda.synchronize()
    STEP_MS[:] = per_step
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


def march_due(cfg, i, last):
    """Whether step i (counted from the first step after setup) repolygonises."""
    return bool((cfg["march_every"] and (i + 1) % cfg["march_every"] == 0)
                or (last and cfg["march_end"]))


def cpu_single(cfg, steps, warm=3, fp64=False, timed=True):
    """The oracle on a single-surface config with the device arm's schedule: setup, `warm`
    untimed steps, then `steps` timed steps (Polys::notify every step, march where the device
    arm marches). Returns (rate, node updates, seconds, surface, polys)."""
    from oracle import oracle as O
    s = O.Surface(cfg["size"], cfg["part"], cfg["L"], fp64=fp64)
    p = O.Polys(s)
    s.seed((0,) * cfg["D"])
    if cfg["expand"]:
        s.run_steps(cfg["expand"], c=-1.0)
    for i in range(warm):
        s.update(**cfg["speed"])
        p.notify()
        if march_due(cfg, i, False):
            p.march()
    nu, secs = 0.0, 0.0
    for i in range(steps):
        nu += s.band_size()
        t0 = time.perf_counter()
        s.update(**cfg["speed"])
        p.notify()
        if march_due(cfg, warm + i, i == steps - 1):
            p.march()
        secs += time.perf_counter() - t0
    return (nu / secs if timed and secs else None), nu, secs, s, p


def cpu_batch(name, cfg, steps, k, shard=0, digest=None):
    """The first k surfaces of a batched config's shard through the oracle for `steps` steps:
    (node updates per second, node updates, seconds). With a list as digest, a hash of each
    surface's final state encoding is appended to it (surfaces the convergence cap dropped:
    None)."""
    from oracle import oracle as O
    sizes, centres, speeds = batch_surfaces(name, cfg, shard)
    items = []
    for sz, c, sp in list(zip(sizes, centres, speeds))[:k]:
        s = O.Surface(sz, cfg["part"], cfg["L"])
        s.seed(c)
        items.append((s, O.Polys(s), sp))
    start = list(items)
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
    if digest is not None:
        import hashlib
        final = {id(s) for s, _, _ in items}
        digest.extend(hashlib.sha1(s.dump().tobytes()).hexdigest() if id(s) in final else None
                      for s, _, _ in start)
    return nu / secs, nu, secs


def cpu_baseline(name, cfg, steps, warm=3):
    threads = cpu_threads()
    if cfg["kind"] == "single":
        rate, nu, secs, _, _ = cpu_single(cfg, steps, warm)
        sample = f"{steps} timed steps after the same setup and {warm} warm-up steps"
    else:
        k = cfg["cpu_subset"]
        rate, nu, secs = cpu_batch(name, cfg, steps, k)
        sample = f"first {k} surfaces of the workload, {steps} steps each, one after another"
    out = {"value": rate, "unit": "node-updates/s", "cores": threads, "kind": "port",
           "sample": f"{sample} ({nu:.3g} node-updates in {secs:.2f} s; the reference's seven "
                     f"parallel loops on {threads} threads)"}
    # a step of a single-surface config is the whole workload's step; a batch config's sample
    # is a subset of its surfaces, so its time is not a step of the workload
    step_ms = secs * 1e3 / steps if cfg["kind"] == "single" and steps else None
    return out, step_ms, nu


def single_config(name, cfg, steps, warmup, node_updates=None):
    """The config object both arms print for a single-surface workload (same keys and values,
    so that the two lines describe the same work)."""
    out = {"workload": cfg["workload"], "name": name, "steps": steps, "warmup": warmup,
           "parallelism": "replicas1"}
    if node_updates is not None:
        out["node_updates"] = int(node_updates)
    return out


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
        if cfg["kind"] != "single":
            steps = min(steps, 10)
        base, step_ms, nu = cpu_baseline(name, cfg, steps, warm=args.warmup)
    if cfg["kind"] == "single":
        config = single_config(name, cfg, steps, args.warmup, nu)
    else:
        config = {"workload": cfg["workload"], "name": name}
    line = {
        "impl": "reference", "metric": metric, "value": base["value"],
        "unit": unit, "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": config,
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# Device arm
# ---------------------------------------------------------------------------------------------

def roofline(fb, make_work, cfg, steps, warm, ms_per_step, node_updates):
    """Roofline of the timed steps, replayed on an identical surface (same setup, warm-up and
    step schedule; the workload is deterministic). Pass A brackets every launch with CUDA events
    on its stream and ranks the kernels by time (shares); pass B brackets only the dominant
    kernel, so its launch durations are not inflated by events around the others. achieved =
    16 B x the work units the kernel processed per launch / its mean launch duration; the
    whole step's fraction (16 B x node updates / the timed step time) is reported beside it."""
    import torch
    hbm, peak_kind = load_peaks()

    def profiled(only):
        work = make_work()
        for i in range(warm):
            work.step(i)
        torch.cuda.synchronize()
        fb.profile_reset()
        fb.profile_only(only)
        fb.profile_enable(True)
        u0 = work.work_units()
        for i in range(steps):
            work.step(warm + i, last=(i == steps - 1))
        torch.cuda.synchronize()
        fb.profile_enable(False)
        fb.profile_only(None)
        prof = fb.profile_read()
        u1 = work.work_units()
        work.close()
        return prof, [b - a for a, b in zip(u0, u1)]

    prof, units = profiled(None)
    tot = sum(v[0] for v in prof.values())
    ranked = sorted(prof.items(), key=lambda kv: -kv[1][0])
    step_s = ms_per_step * steps * 1e-3
    step_achieved = BYTES_PER_NODE_UPDATE * node_updates / step_s / 1e9
    out = {"bound": "hbm", "peak": hbm, "unit": "GB/s", "peak_kind": peak_kind,
           "bytes_per_node_update": BYTES_PER_NODE_UPDATE,
           "step": {"achieved": step_achieved, "frac": step_achieved / hbm,
                    "bytes": BYTES_PER_NODE_UPDATE * node_updates, "seconds": step_s},
           "phase_shares_kernel_ms_per_step": tot / steps,
           "phase_kernels": [[k, round(v[0] / tot, 4), v[1]] for k, v in ranked[:12]],
           "phase_kernels_how": "every phase as its own launch, each bracketed by CUDA events "
                                "(the per-phase path), shares of their summed time"}
    dom = next((k for k, _ in ranked if k in UNIT_OF), None)
    if dom and units[UNIT_OF[dom]]:
        prof_b, _ = profiled(dom)
        ms, nl = prof_b[dom]
        bpl = BYTES_PER_NODE_UPDATE * units[UNIT_OF[dom]] / nl
        achieved = bpl / (ms / nl * 1e-3) / 1e9
        out["phase_kernel"] = {"kernel": dom, "achieved": achieved, "frac": achieved / hbm,
                               "bytes_per_launch": bpl, "avg_launch_us": 1e3 * ms / nl,
                               "ms_per_step": ms / steps, "launches": nl}
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            try:
                tj = json.load(open(tf))
                t = tj.get(dom)
                if t:
                    out["phase_kernel"]["traffic"] = t["bytes_per_unit"] * units[UNIT_OF[dom]] / nl
            except Exception:
                pass
    if "phase_kernel" in out:
        pk = out["phase_kernel"]
        out.update({"kernel": pk["kernel"], "achieved": pk["achieved"], "frac": pk["frac"],
                    "traffic": pk.get("traffic"), "bytes_per_launch": pk["bytes_per_launch"],
                    "avg_launch_us": pk["avg_launch_us"], "kernel_ms_per_step": pk["ms_per_step"],
                    "launches": pk["launches"], "share_of_step": pk["ms_per_step"] / ms_per_step})
    return out


def capture_single(work):
    """The device state after the timed steps, for the parity check against the oracle."""
    s, p = work.s, work.p
    n = s.partitions()[0]
    vtx, spx, counts = p.gather(range(n))
    return {"dump": s.dump(), "snapshot": s.snapshot(), "changes": p.changes(),
            "totals": p.totals(), "vtx": vtx, "spx": spx, "counts": counts}


def single_parity(cfg, dev, o, op, o64, op64):
    """Device state against the oracle run of the same steps (bit-exact lists, orders,
    partition lists and simplices; values and vertices within 1e-5), and its error against the
    FP64 run of the same method."""
    import numpy as np
    from oracle import oracle as O
    from tests.dumps import first_difference
    diff = first_difference(dev["dump"], o.dump())
    phi_err = float(np.abs(dev["snapshot"] - o.snapshot()).max())
    n = o.partitions()[0]
    poly_ok, vtx_err, pairs = True, 0.0, []
    v0 = s0 = 0
    for pc in range(n):
        nv, ns = (int(x) for x in dev["counts"][pc])
        gv, gs = dev["vtx"][v0:v0 + nv], dev["spx"][s0:s0 + ns]
        v0, s0 = v0 + nv, s0 + ns
        ov, os_, _ = op.partition(pc)
        if gs.shape != os_.shape or not np.array_equal(gs, os_):
            poly_ok = False
        elif ov.size:
            vtx_err = max(vtx_err, float(np.abs(gv - ov).max()))
        pairs.append((gv, gs, op64.partition64(pc), op64.partition(pc)[1]))
    fp64 = O.fp64_errors(dev["snapshot"], o64.snapshot64(), cfg["L"], pairs)
    ok = diff is None and phi_err <= 1e-5 and poly_ok and vtx_err <= 1e-5 and \
        list(dev["changes"]) == list(op.changes())
    return {"matches_oracle": ok, "first_difference": diff, "phi_max_abs_vs_oracle": phi_err,
            "simplices_equal": poly_ok, "vertex_max_abs_vs_oracle": vtx_err,
            "tolerance": 1e-5, "fp64": fp64,
            "how": "device state after the timed steps against the oracle port run of the same "
                   "setup, warm-up and steps (the CPU baseline run), and against the oracle's "
                   "FP64 run of the same method"}


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


def serve_budget(cfg):
    """The brick-pool budget of the served config, less what the device cannot spare (the pool
    is allocated up front; 8 GB stay free for the partition tables, arenas and the rest)."""
    import torch
    free, _ = torch.cuda.mem_get_info()
    return min(cfg["budget"], max(1e9, free - 8e9 - 2e9 * cfg["slots"] / 512))


def serve_one_rate(srv, cfg, lam, shard=0, stream=None):
    """Feeds one rate's stream into the server in real time (arrival = the scheduled time on
    the server's clock); latency (arrival to result) and throughput figures."""
    stream = serve_requests(cfg, lam, shard) if stream is None else stream
    st0 = srv.stats()
    t_first = srv.now()
    for off, req in stream:
        due = t_first + off
        while srv.now() < due:
            time.sleep(min(0.0005, max(0.0, due - srv.now())))
        req.arrival = due
        srv.submit(req)
    if not srv.drain(timeout=900):
        raise RuntimeError("serving did not drain")
    ids = {req.rid for _, req in stream}
    res = [r for r in srv.results() if r.rid in ids]
    st = srv.stats()
    t_end = max((r.done for r in res), default=t_first)
    lat = sorted(r.latency for r in res)
    pct = (lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] * 1e3) if lat else (lambda q: None)
    nu = st["node_updates"] - st0["node_updates"]
    steps = st["steps"] - st0["steps"]
    return {"lambda_per_s": lam, "requests": len(stream),
            "admitted": st["admitted"] - st0["admitted"],
            "rejected": st["rejected"] - st0["rejected"], "stopped": sum(r.stopped for r in res),
            "p50_ms": pct(0.50), "p99_ms": pct(0.99), "mean_ms": 1e3 * sum(lat) / max(len(lat), 1),
            "node_updates_per_s": nu / max(t_end - t_first, 1e-9), "node_updates": nu,
            "seconds": t_end - t_first, "batched_steps": steps,
            "mean_in_flight": sum((r.done - r.admitted) for r in res) / max(t_end - t_first,
                                                                             1e-9),
            "peak_reserved_gb": st["peak_reserved_bricks"] * srv.brick_bytes / 1e9,
            "peak_used_gb": st["peak_used_bricks"] * srv.brick_bytes / 1e9}


def serve_plain(fb, cfg, k):
    """The plain path on the first k requests of the 1k/s stream: one Surface (+ Polys) per
    request, one request after another, wall clock from the seed to the result (the request's
    updates, its polygonisation when asked, the node-update count read back). Surface
    construction is timed apart. Returns (rate, node updates, seconds, construction seconds)."""
    reqs = [r for _, r in serve_requests(cfg, 1000)[:k]]
    nu, secs, make = 0, 0.0, 0.0
    for r in reqs:
        t0 = time.perf_counter()
        s = fb.Surface(r.size, cfg["part"], cfg["L"], **TUNING)
        p = fb.Polys(s)
        t1 = time.perf_counter()
        s.seed(r.centre)
        for _ in range(r.steps):
            try:
                s.update(**r.speed)
            except fb.FeltError:  # stopped: its convergence loop did not terminate
                break
            p.notify()
        if r.polys:
            p.march()
            p.totals()
        n = s.node_updates()
        t2 = time.perf_counter()
        make += t1 - t0
        secs += t2 - t1
        nu += n
        p.close()
        s.close()
    return nu / secs, nu, secs, make


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
    from felt_b200.serving import Server
    budget = serve_budget(cfg)
    srv = Server(layers=cfg["L"], part=cfg["part"], budget_bytes=budget, slots=cfg["slots"],
                 max_size=cfg["max_size"])
    try:
        # warm-up: a few requests through every code path (graph captures, arenas)
        serve_one_rate(srv, cfg, 1000, shard=rank,
                       stream=[(t, r) for t, r in serve_requests(cfg, 1000, shard=rank + 99)[:16]])
        clocks = ClockSampler(local)
        clocks.start()
        l0 = fb.launch_count()
        sweep = [serve_one_rate(srv, cfg, lam, shard=rank) for lam in cfg["lambdas"]]
        launches = fb.launch_count() - l0
        clk = clocks.stop()
    finally:
        srv.close()
    best = max(sweep, key=lambda r: r["node_updates_per_s"])
    value = best["node_updates_per_s"]
    if pg:
        secs, _, nu = combine_ranks(pg, best["seconds"], 0.0, best["node_updates"], "cuda")
        value = nu / secs
    extra = {}
    cpu = None
    if rank == 0:
        p_rate, _, _, _ = serve_plain(fb, cfg, cfg["plain_subset"])
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
    step_ms = sorted(STEP_MS)
    clk = clocks.stop()
    if pg:
        t_ms, wall_s, nu = combine_ranks(pg, t_ms, wall_s, nu, "cuda")
    value = nu / (t_ms / 1e3)
    import ctypes as C
    e2e = {"value": nu / wall_s, "unit": "node-updates/s",
           "h2d_bytes_per_step": C.sizeof(fb.Speed) * (cfg.get("n") or 1),
           "d2h_bytes_per_step": d2h // steps}

    extra = {}
    roof = cpu = parity = batched = batched_2d = served = None
    dev_state = None
    single = cfg["kind"] == "single"
    if rank == 0 and single and ws == 1 and not args.no_cpu:
        dev_state = capture_single(work)
    work.close()
    del flush
    if rank == 0:
        def make_work():
            return (SingleWork(fb, cfg, args.brick_capacity) if single
                    else BatchWork(fb, cfg, name, shard=rank))
        roof = roofline(fb, make_work, cfg, steps, args.warmup, t_ms / steps, nu)
        if cfg["kind"] == "batch" and not args.no_plain:
            extra["plain_comparison"] = measure_batched(fb, name, min(steps, 20), args.warmup)
        if name == "c2" and not args.no_extras:
            # the headline metric's other halves, on the same GPU in the same run: the batched
            # 3D workload against the plain path, and the served request mix
            batched = measure_batched(fb, "c4", 20, 3)
            batched_2d = measure_batched(fb, "c3", 20, 3)
            served = measure_served(fb, "c5", (300, 1000, 3000))
    if rank == 0 and ws == 1 and not args.no_cpu:
        if single:
            threads = cpu_threads()
            rate, cnu, secs, o, op = cpu_single(cfg, steps, args.warmup)
            cpu = {"value": rate, "unit": "node-updates/s", "cores": threads, "kind": "port",
                   "sample": f"the same {steps} timed steps after the same setup and "
                             f"{args.warmup} warm-up steps ({cnu:.3g} node-updates in "
                             f"{secs:.2f} s; the reference's seven parallel loops on {threads} "
                             f"threads)"}
            _, _, _, o64, op64 = cpu_single(cfg, steps, args.warmup, fp64=True, timed=False)
            parity = single_parity(cfg, dev_state, o, op, o64, op64)
            parity["oracle_node_updates_equal"] = int(cnu) == int(nu)
            del o, op, o64, op64, dev_state
        else:
            cpu, _, _ = cpu_baseline(name, cfg, cfg["cpu_steps"])

    if rank == 0:
        if single:
            config = single_config(name, cfg, steps, args.warmup, nu)
        else:
            config = {"workload": cfg["workload"], "name": name,
                      "parallelism": f"surface shards x{ws} (independent surfaces per rank)",
                      "node_updates": nu}
        config.update(extra)
        line = {
            "metric": "narrow-band node-updates/s", "value": value, "unit": "node-updates/s",
            "n_gpus": ws, "steps": steps, "warmup": args.warmup, "ms_per_step": t_ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config,
            "timing": {"l2": "flushed between timed steps (256 MB write)",
                       "value": "device time of the timed steps (CUDA events on the surface's "
                                "stream), inputs resident",
                       "e2e": "wall clock through the C ABI with the speed going in and the "
                              "step's result (band size; the re-marched polygons on march "
                              "steps) coming out each step",
                       "step_ms": {"min": step_ms[0], "median": step_ms[len(step_ms) // 2],
                                   "max": step_ms[-1]} if step_ms else None},
            "roofline": roof, "cpu_baseline": cpu, "parity": parity,
            "batched": batched, "batched_2d": batched_2d, "served": served,
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
    ap.add_argument("--no-extras", action="store_true",
                    help="default config only: skip the batched and served measurements")
    ap.add_argument("--brick-capacity", type=int, default=0,
                    help="brick pool capacity of single-surface configs (0 = automatic)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop")
    ap.add_argument("--launch-mode", type=int, default=0, choices=[0, 1, 2],
                    help="fg_config.launch_mode: 1 one CUDA graph per update (0 = automatic = "
                         "1), 2 every kernel launched from the host (per-kernel profilers)")
    ap.add_argument("--autotune", action="store_true",
                    help="launch shapes by measurement (fg_autotune) instead of by brick size")
    ap.add_argument("--delta-kernel", type=int, default=0, choices=[0, 1, 2],
                    help="fg_config.delta_kernel: the curvature speed functor 1 reading the pool "
                         "directly, 2 over bricks staged with their halo (0 = automatic)")
    ap.add_argument("--fuse-passes", type=int, default=0, choices=[0, 1, 2, 3],
                    help="fg_config.fuse_passes: the distance passes 1 as 4L launches, 2 as 2L+1 "
                         "fused ones, 3 tiled per brick in shared memory (0 = automatic)")
    ap.add_argument("--dist-split", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="fg_config.dist_split: warps per partition entry in the first distance "
                         "pass (0 = automatic)")
    ap.add_argument("--record-passes", type=int, default=0, choices=[0, 1, 2],
                    help="fg_config.record_passes: 1 a warp, 2 a block per partition entry in the "
                         "passes that record status changes (0 = automatic)")
    args = ap.parse_args()
    TUNING.update(launch_mode=args.launch_mode, autotune=args.autotune,
                  delta_kernel=args.delta_kernel, fuse_passes=args.fuse_passes,
                  dist_split=args.dist_split, record_passes=args.record_passes)
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
