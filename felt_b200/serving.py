"""Serving many independent level-set requests on one GPU: a thin client of the fg_server_* C ABI.

A request is one Surface<D,L> job: grid size, seed position, builtin speed, number of global
updates, and whether to polygonise the result. The reference runs one surface at a time; the
server (libfelt_gpu.so, fg_server.cu) batches them continuously: one long-lived pool of
`slots` surfaces sharing one brick pool, advanced together one Surface::update per step by a
worker thread, with requests that arrive while others run taking freed slots at the next step
boundary. Each result equals a separate Surface run alone on the same request.

Admission is by the brick pool: a request reserves the bricks its band can reach and is
rejected at submission when the reservations in flight and queued would exceed the pool
(budget_bytes of device memory, or brick_capacity bricks).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import FeltError, Speed, _chk, lib, make_speed

ERR_CAPACITY = -13
ERR_TIMEOUT = -14


class _Config(C.Structure):
    _fields_ = [("dims", C.c_int), ("layers", C.c_int), ("part", C.c_int * 3),
                ("max_size", C.c_int * 3), ("slots", C.c_size_t),
                ("brick_capacity", C.c_size_t), ("budget_bytes", C.c_double),
                ("vertex_capacity", C.c_size_t), ("keep_outputs", C.c_int),
                ("reserved", C.c_int * 7)]


class _Request(C.Structure):
    _fields_ = [("size", C.c_int * 3), ("centre", C.c_int * 3), ("speed", Speed),
                ("steps", C.c_int), ("polygonise", C.c_int), ("tag", C.c_uint64)]


class _Result(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int), ("steps_done", C.c_int),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("node_updates", C.c_ulonglong), ("vertices", C.c_ulonglong),
                ("simplices", C.c_ulonglong)]


class _Stats(C.Structure):
    _fields_ = [(k, C.c_ulonglong) for k in (
        "submitted", "admitted", "rejected", "started", "completed", "failed", "steps",
        "node_updates", "capacity_bricks", "reserved_bricks", "peak_reserved_bricks",
        "peak_used_bricks", "queued", "in_flight")] + [("fault_code", C.c_int),
                                                       ("reserved", C.c_int * 7)]


@dataclass
class Request:
    size: tuple            # grid size
    centre: tuple          # seed position
    speed: dict            # dict(c=, a=, n=, seed=) as for Surface.update
    steps: int             # global updates
    polys: bool            # polygonise after the last update
    kind: str = "constant"
    arrival: float = 0.0   # seconds on the server clock (set by the caller, else submission)
    rid: int = -1


@dataclass
class Result:
    rid: int
    arrival: float
    done: float            # seconds on the server clock when the result was ready
    stopped: bool = False  # the update's convergence loop did not settle (surface stopped)
    dump: object = None    # the surface's state encoding (fg_dump), when the server keeps it
    admitted: float = 0.0  # when it took a slot
    status: int = 0
    steps_done: int = 0
    node_updates: int = 0
    vertices: int = 0
    simplices: int = 0

    @property
    def latency(self):
        return self.done - self.arrival


def _as_request(req: Request, D):
    r = _Request()
    for a in range(D):
        r.size[a] = int(req.size[a])
        r.centre[a] = int(req.centre[a])
    r.speed = make_speed(**req.speed)
    r.steps = int(req.steps)
    r.polygonise = 1 if req.polys else 0
    r.tag = int(req.rid)
    return r


def reserve_bricks(req: Request, L, part):
    """The bricks a server with this layer count and partition shape reserves for a request
    (its admission bound; fg_request_bricks, host arithmetic only)."""
    D = len(part)
    cfg = _Config()
    cfg.dims, cfg.layers = D, int(L)
    for a in range(D):
        cfg.part[a] = int(part[a])
    n = C.c_ulonglong()
    _chk(lib().fg_request_bricks(C.byref(cfg), C.byref(_as_request(req, D)), C.byref(n)))
    return n.value


def brick_bytes(L, part):
    """Device bytes of one brick of the pool (fg_brick_bytes)."""
    v = C.c_double()
    _chk(lib().fg_brick_bytes(len(part), int(L), (C.c_int * len(part))(*part), C.byref(v)))
    return v.value


class Server:
    """Continuous-batching level-set server (fg_server_*).

    submit() admits or rejects a request at its arrival; results() returns the finished ones.
    With keep_outputs each result carries its surface's final state encoding, and polys(rid)
    its polygons."""

    def __init__(self, layers=2, part=(8, 8, 8), budget_bytes=150e9, slots=256,
                 max_size=(256, 256, 256), keep_outputs=False, brick_capacity=0,
                 vertex_capacity=0):
        self.D = len(part)
        self.L = int(layers)
        self.part = tuple(int(p) for p in part)
        self.keep_outputs = bool(keep_outputs)
        cfg = _Config()
        cfg.dims, cfg.layers = self.D, self.L
        for a in range(self.D):
            cfg.part[a] = self.part[a]
            cfg.max_size[a] = int(max_size[a])
        cfg.slots = int(slots)
        cfg.brick_capacity = int(brick_capacity)
        cfg.budget_bytes = float(budget_bytes)
        cfg.vertex_capacity = int(vertex_capacity)
        cfg.keep_outputs = 1 if keep_outputs else 0
        h = C.c_void_p()
        _chk(lib().fg_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._requests = {}
        self._results = []
        self.brick_bytes = brick_bytes(self.L, self.part)

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None:
            lib().fg_server_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def now(self):
        t = C.c_double()
        _chk(lib().fg_server_now(self._h, C.byref(t)))
        return t.value

    def submit(self, req: Request):
        """Admit (True) or reject (False) a request at its arrival."""
        rc = lib().fg_server_submit(self._h, C.byref(_as_request(req, self.D)))
        if rc == ERR_CAPACITY:
            return False
        _chk(rc)
        self._requests[int(req.rid)] = req
        return True

    def request_bricks(self, req: Request):
        """The bricks the server reserves for a request."""
        return reserve_bricks(req, self.L, self.part)

    def _poll(self, wait_s=0.0):
        buf = (_Result * 256)()
        n = C.c_size_t()
        got = 0
        while True:
            _chk(lib().fg_server_poll(self._h, buf, C.c_size_t(256), C.byref(n),
                                      C.c_double(wait_s if not got else 0.0)))
            for i in range(n.value):
                self._results.append(self._convert(buf[i]))
            got += n.value
            if n.value < 256:
                return got

    def _convert(self, r):
        req = self._requests.pop(int(r.tag), None)
        arrival = req.arrival if req is not None and req.arrival > 0 else r.t_submit
        dump = None
        if self.keep_outputs and r.status in (0, ERR_TIMEOUT):
            dump = self._kept_dump(int(r.tag))
        return Result(int(r.tag), arrival, r.t_done, r.status == ERR_TIMEOUT, dump,
                      r.t_admit, r.status, r.steps_done, r.node_updates, r.vertices,
                      r.simplices)

    def _kept_dump(self, tag):
        n = C.c_size_t()
        _chk(lib().fg_server_result_dump(self._h, C.c_uint64(tag), None, C.c_size_t(0),
                                         C.byref(n)))
        out = np.zeros(max(1, n.value), dtype=np.uint32)
        _chk(lib().fg_server_result_dump(self._h, C.c_uint64(tag),
                                         out.ctypes.data_as(C.POINTER(C.c_uint32)),
                                         C.c_size_t(out.size), C.byref(n)))
        return out[: n.value]

    def polys(self, rid):
        """A kept result's polygons: per partition (vertices (nv, per), simplices (ns, D))."""
        nv, ns, npt = C.c_size_t(), C.c_size_t(), C.c_size_t()
        tag = C.c_uint64(int(rid))
        _chk(lib().fg_server_result_polys(self._h, tag, None, 0, None, 0, None, 0, C.byref(nv),
                                          C.byref(ns), C.byref(npt)))
        per = 2 * self.D if self.D == 3 else self.D
        vtx = np.zeros(max(1, nv.value * per), dtype=np.float32)
        spx = np.zeros(max(1, ns.value * self.D), dtype=np.uint32)
        cnt = np.zeros(max(1, 2 * npt.value), dtype=np.uint32)
        _chk(lib().fg_server_result_polys(self._h, tag, vtx.ctypes.data_as(C.POINTER(C.c_float)),
                                          C.c_size_t(vtx.size),
                                          spx.ctypes.data_as(C.POINTER(C.c_uint32)),
                                          C.c_size_t(spx.size),
                                          cnt.ctypes.data_as(C.POINTER(C.c_uint32)),
                                          C.c_size_t(cnt.size), C.byref(nv), C.byref(ns),
                                          C.byref(npt)))
        out, v0, s0 = [], 0, 0
        for p in range(npt.value):
            a, b = int(cnt[2 * p]), int(cnt[2 * p + 1])
            out.append((vtx[v0 * per:(v0 + a) * per].reshape(a, per),
                        spx[s0 * self.D:(s0 + b) * self.D].reshape(b, self.D)))
            v0 += a
            s0 += b
        return out

    def stats(self):
        st = _Stats()
        _chk(lib().fg_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _Stats._fields_ if k != "reserved"}

    def drain(self, timeout=600.0):
        """Waits until every admitted request has finished."""
        t_end = time.perf_counter() + timeout
        while time.perf_counter() < t_end:
            self._poll(0.05)
            st = self.stats()
            if st["fault_code"]:
                raise FeltError(st["fault_code"], "serving worker failed")
            if st["completed"] + st["failed"] >= st["admitted"] and not st["queued"] \
                    and not st["in_flight"]:
                self._poll(0.0)
                return True
        return False

    def results(self):
        self._poll(0.0)
        return list(self._results)

    @property
    def admitted(self):
        return self.stats()["admitted"]

    @property
    def rejected(self):
        return self.stats()["rejected"]

    @property
    def node_updates(self):
        return self.stats()["node_updates"]
