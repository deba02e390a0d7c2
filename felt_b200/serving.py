"""Serving many independent level-set requests on one GPU.

A request is one Surface<3,L> job: grid size, seed position, speed, number of global updates,
and whether to polygonise the result. The reference runs one surface at a time; here requests
that arrive close together form a *wave*: one Batch whose surfaces advance in the same kernel
launches. A wave runs on its own worker thread and CUDA stream, so several waves overlap on the
GPU. Requests in a wave may ask for different step counts: a request that has had its last
update (and, if asked, its polygonisation) is paused, so later launches skip it and its state
stays exactly what a separate Surface given the same updates would hold.

Admission is by device memory: each request reserves an upper bound of the brick-pool bytes it
can reach (partitions within reach of its band after its steps, at the worst speed its kind
allows), and a request that would push the reserved total over the budget is rejected at
arrival. Reservations are returned when the request's wave ends.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass

from . import Batch

# Largest |delta| per update for each builtin speed kind of a request (bounds the band's reach).
_VMAX = {"constant": 0.6, "curvature": 0.8, "noise": 0.4}


@dataclass
class Request:
    size: tuple            # grid size (3 ints)
    centre: tuple          # seed position
    speed: dict            # dict(c=, a=, n=, seed=) as for Batch.update
    steps: int             # global updates
    polys: bool            # polygonise after the last update
    kind: str = "constant"
    arrival: float = 0.0   # seconds on the server clock
    rid: int = -1


@dataclass
class Result:
    rid: int
    arrival: float
    done: float            # seconds on the server clock when the result was ready
    stopped: bool = False  # the update's convergence loop did not settle (surface stopped)
    dump: object = None    # the surface's state encoding (fg_dump), when the server keeps it

    @property
    def latency(self):
        return self.done - self.arrival


def brick_bytes(L, part):
    """Device bytes of one brick slot: phi, delta, lookup, 2L+1 lists, status, status lists, two
    affected buffers, expansion claims (per leaf), as the engine allocates them."""
    nl = 2 * L + 1
    bv = math.prod(part)
    return bv * (4 + 4 + 2 + 2 * nl + 1 + 2 * nl + 2 * 2 + 2 * 2 * nl + 8) + 4 * (3 * nl + 6)


def partition_bytes(L):
    """Device bytes per partition of a grid (lists, lookups, flags), engine and polygoniser."""
    nl = 2 * L + 1
    return 4 * (12 * nl + 24)


def reserve_bytes(req: Request, L, part):
    """Upper bound of the device bytes a request can occupy: every partition that the band can
    reach within its steps holds a brick (the ball of radius 1 + steps * vmax + L + 1 around the
    seed, by its bounding box, clipped to the grid), plus the grid's partition-level arrays."""
    reach = 1.0 + req.steps * _VMAX.get(req.kind, 1.0) + L + 1
    nb = 1
    npart = 1
    for a in range(3):
        span = min(req.size[a], int(math.ceil(2 * reach)) + 1)
        nb *= min(-(-req.size[a] // part[a]) + 1, -(-span // part[a]) + 1)
        npart *= -(-req.size[a] // part[a]) + 1
    return nb, nb * brick_bytes(L, part) + npart * partition_bytes(L)


@dataclass
class _Wave:
    reqs: list
    bricks: int
    bytes: int


class Server:
    """Poisson-fed request server over batched surfaces.

    submit() admits or rejects a request at its arrival; a scheduler thread groups the admitted
    requests into waves every `tick` seconds and hands each wave to a worker (at most `workers`
    waves in flight). results() returns the finished requests; with keep_outputs each result
    carries its surface's final state encoding."""

    def __init__(self, layers=2, part=(8, 8, 8), budget_bytes=150e9, workers=4, tick=0.002,
                 max_wave=512, keep_outputs=False):
        self.L = layers
        self.keep_outputs = keep_outputs
        self.part = tuple(part)
        self.budget = float(budget_bytes)
        self.tick = tick
        self.max_wave = max_wave
        self.t0 = time.perf_counter()
        self._lock = threading.Lock()
        self._reserved = 0.0
        self._pending = []
        self._results = []
        self._errors = []
        self.admitted = 0
        self.rejected = 0
        self.node_updates = 0  # band nodes processed by the finished waves
        self._waves = queue.Queue()
        self._stop = threading.Event()
        self._inflight = threading.Semaphore(workers)
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(workers)]
        self._sched = threading.Thread(target=self._schedule, daemon=True)
        for w in self._workers:
            w.start()
        self._sched.start()

    def now(self):
        return time.perf_counter() - self.t0

    def submit(self, req: Request):
        """Admit (True) or reject (False) a request at its arrival."""
        _, need = reserve_bytes(req, self.L, self.part)
        with self._lock:
            if self._reserved + need > self.budget:
                self.rejected += 1
                return False
            self._reserved += need
            self.admitted += 1
            self._pending.append(req)
        return True

    def _schedule(self):
        while not self._stop.is_set():
            time.sleep(self.tick)
            with self._lock:
                take, self._pending = self._pending[:self.max_wave], self._pending[self.max_wave:]
            if not take:
                continue
            self._inflight.acquire()
            nb = sum(reserve_bytes(r, self.L, self.part)[0] for r in take)
            by = sum(reserve_bytes(r, self.L, self.part)[1] for r in take)
            self._waves.put(_Wave(take, nb, by))

    def _work(self):
        while True:
            w = self._waves.get()
            if w is None:
                return
            try:
                self._run_wave(w)
            except Exception as e:  # recorded, the server keeps serving
                self._errors.append(repr(e))
            finally:
                with self._lock:
                    self._reserved -= w.bytes
                self._inflight.release()

    def _run_wave(self, w: _Wave):
        reqs = w.reqs
        b = Batch([r.size for r in reqs], self.part, self.L, brick_capacity=max(w.bricks, 1))
        try:
            b.seed([r.centre for r in reqs])
            speeds = b.speed_array([r.speed for r in reqs])
            nu = 0
            for step in range(1, max(r.steps for r in reqs) + 1):
                b.update(speeds)
                b.polys_notify()
                finishing = [i for i, r in enumerate(reqs) if r.steps == step]
                if not finishing:
                    continue
                if any(reqs[i].polys for i in finishing):
                    b.polys_march()
                nu = b.node_updates()  # synchronises the wave's stream: results are ready
                t = self.now()
                out = [Result(reqs[i].rid, reqs[i].arrival, t, b.stopped(i),
                              b.dump(i) if self.keep_outputs else None) for i in finishing]
                for i in finishing:
                    b.pause(i)
                with self._lock:
                    self._results.extend(out)
            with self._lock:
                self.node_updates += nu
        finally:
            b.close()

    def drain(self, timeout=600.0):
        """Waits until every admitted request has finished."""
        t_end = time.perf_counter() + timeout
        while time.perf_counter() < t_end:
            with self._lock:
                n = len(self._results)
                busy = self._pending or self._reserved > 0
            if n >= self.admitted and not busy:
                return True
            if self._errors:
                raise RuntimeError("serving worker failed: " + self._errors[0])
            time.sleep(0.002)
        return False

    def close(self):
        self._stop.set()
        self._sched.join(timeout=5)
        for _ in self._workers:
            self._waves.put(None)
        for w in self._workers:
            w.join(timeout=60)

    def results(self):
        return list(self._results)

    @property
    def errors(self):
        return list(self._errors)
