"""Benchmark of the sparse-field level-set hot path (Surface<D,L>::update + Polys) on B200.

Workload (default, --config c2): Surface<3,3> float32, 512^3 isogrid with 16^3 partitions,
seeded at the origin and expanded to radius ~100 with 100 untimed steps of speed -1, then timed
steps of delta = -0.2*curv(pos) + 0.1*h(pos, 1234) (h = hashed uniform [-1,1) noise), with
Polys::notify every step and Polys::march every 10th step. A "step" is one Surface::update plus
that repolygonisation. Metric: narrow-band node-updates/s (band size at each step's start).

Arms:
  default           the device engine (libfelt_gpu.so) driven through its C ABI.
  --impl reference  the reference algorithm's CPU implementation (the oracle port, compiled
                    from oracle/), on the same workload and metric, bounded sample.

Prints ONE JSON line on rank 0. Multi-GPU (torchrun): every rank advances its own independent
surface (replicas; a single surface does not shard), value = all ranks' node-updates / the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (D, L, size, part, expansion steps, timed speed, march every)
    "c2": dict(D=3, L=3, size=(512, 512, 512), part=(16, 16, 16), expand=100,
               speed=dict(a=-0.2, n=0.1, seed=1234), march_every=10,
               workload="Surface<3,3> 512^3 / 16^3 partitions, r~100, "
                        "speed -0.2*curv + 0.1*hash_noise, repolygonise every 10 steps"),
    "c1": dict(D=3, L=2, size=(64, 64, 64), part=(8, 8, 8), expand=0,
               speed=dict(c=-0.5), march_every=0,
               workload="Surface<3,2> 64^3 / 8^3 partitions, speed -0.5"),
}

# Algorithmic bytes per work unit of the kernels whose roofline is reported:
#  k_dist1: per band node of the layer: 2 B list index + 4 B phi read + 4 B delta write.
#  k_dist2: per band node: 2 B list index + 4 B delta read + 4 B phi write.
#  k_delta_builtin: per zero-layer node: 2 B index + 4 B phi + 4 B delta write.
#  k_flush_leaf: per leaf edit: 2 B status entry + 1 B to-layer + 2 B lookup read + 2 B list
#                write + 2 B lookup write + 4 B swap-in (moved entry and its lookup).
#  k_polys_march: per cell: 2 B leaf index + 4 B phi (corners are neighbours' phi).
UNIT_BYTES = {"k_dist1": (0, 10), "k_dist2": (0, 10), "k_delta_builtin": (1, 10),
              "k_delta_smem": (1, 10), "k_flush_smem": (2, 13),
              "k_flush_leaf": (2, 13), "k_polys_march": (3, 6)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

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
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(cfg, steps, warm=3):
    """The oracle port on a bounded sample of the same workload: the same setup (seed and
    expansion), then `steps` timed steps of the same speed with the same repolygonisation.
    Returns (node-updates/s, sample description)."""
    from oracle import oracle as O
    s = O.Surface(cfg["size"], cfg["part"], cfg["L"])
    p = O.Polys(s)
    s.seed((0,) * cfg["D"])
    if cfg["expand"]:
        s.run_steps(cfg["expand"], c=-1.0)
    for _ in range(warm):
        s.update(**cfg["speed"])
        p.notify()
    nu = 0.0
    secs = 0.0
    for i in range(steps):
        nu += s.band_size()
        t0 = time.perf_counter()
        s.update(**cfg["speed"])
        p.notify()
        if cfg["march_every"] and (i + 1) % cfg["march_every"] == 0:
            p.march()
        secs += time.perf_counter() - t0
    return nu / secs, nu, secs


def run_reference(args, cfg):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O  # noqa: F401  (builds liboracle.so if missing)
    steps = args.steps
    for _ in range(args.warmup):
        pass
    rate, nu, secs = cpu_baseline(cfg, steps)
    line = {
        "impl": "reference",
        "metric": "narrow-band node-updates/s", "value": rate, "unit": "node-updates/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / max(steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "steps_timed": steps},
        "cpu_baseline": {"value": rate, "unit": "node-updates/s", "cores": 1, "kind": "port",
                         "sample": f"{steps} steps of the timed speed after the same setup"},
        "e2e": {"value": rate, "unit": "node-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_felt(args, cfg):
    import torch
    import felt_b200 as fb

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        pg = dist

    D = cfg["D"]
    s = fb.Surface(cfg["size"], cfg["part"], cfg["L"])
    p = fb.Polys(s)
    s.seed((0,) * D)
    for _ in range(cfg["expand"]):
        s.update(c=-1.0)
    stream = torch.cuda.ExternalStream(s.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(i):
        s.update(**cfg["speed"])
        p.notify()
        if cfg["march_every"] and (i + 1) % cfg["march_every"] == 0:
            p.march()

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    nu0 = s.node_updates()
    l0 = fb.launch_count()
    total_ms = 0.0
    for i in range(args.steps):
        flush.fill_(float(i))  # L2 flush (256 MB > 126 MB L2) between timed steps, untimed
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step(i)
        b.record(stream)
        b.synchronize()
        total_ms += a.elapsed_time(b)
    torch.cuda.synchronize()
    launches = fb.launch_count() - l0
    nu = s.node_updates() - nu0
    clk = clocks.stop()
    t_ms = total_ms
    if pg:
        tt = torch.tensor([t_ms, float(nu)], dtype=torch.float64, device="cuda")
        mx = tt.clone()
        pg.all_reduce(mx[:1], op=pg.ReduceOp.MAX)
        pg.all_reduce(tt[1:], op=pg.ReduceOp.SUM)
        t_ms = float(mx[0])
        nu = float(tt[1])
    value = nu / (t_ms / 1e3)

    # ---- end to end through the C ABI with host buffers ----
    import ctypes as C
    lib = fb.lib()
    e2e_steps = max(3, min(args.steps, 20))
    h2d = C.sizeof(fb.Speed)
    d2h = 0
    e2e_s = 0.0
    e2e_nu = 0
    for i in range(e2e_steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n0 = s.node_updates()
        sp = fb.make_speed(**cfg["speed"])
        fb._chk(lib.fg_update_builtin(s._h, C.byref(sp)))
        p.notify()
        if cfg["march_every"] and (i + 1) % cfg["march_every"] == 0:
            p.march()
            for part in p.changes():
                vtx, spx, _ = p.partition(part)
                d2h += vtx.nbytes + spx.nbytes
        n1 = s.node_updates()
        d2h += 16
        e2e_s += time.perf_counter() - t0
        e2e_nu += n1 - n0
    e2e = {"value": e2e_nu / e2e_s, "unit": "node-updates/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h // e2e_steps}

    # ---- per-kernel device times for the roofline (separate pass, profiling on) ----
    roof = None
    if rank == 0:
        units0 = s.work_units()
        fb.profile_reset()
        fb.profile_enable(True)
        nprof = max(cfg["march_every"] or 5, 10)
        for i in range(nprof):
            step(i)
        torch.cuda.synchronize()
        fb.profile_enable(False)
        prof = fb.profile_read()
        units1 = s.work_units()
        tot = sum(v[0] for v in prof.values())
        ranked = sorted(prof.items(), key=lambda kv: -kv[1][0])
        hbm, peak_kind = load_peaks()
        dom = next((k for k, _ in ranked if k in UNIT_BYTES), None)
        if dom:
            ms, nl = prof[dom]
            ui, per = UNIT_BYTES[dom]
            units = units1[ui] - units0[ui]
            bytes_per_launch = per * units / nl
            achieved = bytes_per_launch / (ms / nl * 1e-3) / 1e9
            roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                    "traffic": None, "bytes_per_launch": bytes_per_launch,
                    "avg_launch_us": 1e3 * ms / nl,
                    "share_of_step_kernel_time": prof[dom][0] / tot if tot else None,
                    "top_kernels": [[k, round(v[0] / tot, 4), v[1]] for k, v in ranked[:8]]}
            tf = os.path.join(ROOT, "profiles", "traffic.json")
            if os.path.exists(tf):
                try:
                    t = json.load(open(tf)).get(dom)
                    if t:
                        roof["traffic"] = t["bytes_per_unit"] * units / nl
                except Exception:
                    pass

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        rate, cnu, csecs = cpu_baseline(cfg, args.cpu_steps)
        cpu = {"value": rate, "unit": "node-updates/s", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_steps} timed steps after the same seed+expansion setup "
                         f"({cnu:.3g} node-updates in {csecs:.2f} s, single thread)"}

    if rank == 0:
        line = {
            "metric": "narrow-band node-updates/s", "value": value, "unit": "node-updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "parallelism": f"replicas{ws}",
                       "l2": "flushed between timed steps (256 MB write)",
                       "node_updates": nu},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="felt", choices=["felt", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_felt(args, cfg)


if __name__ == "__main__":
    main()
