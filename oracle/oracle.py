"""ctypes wrapper over the CPU oracle library (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker. The product (felt_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


class Speed(C.Structure):
    _fields_ = [("kind", C.c_int), ("c", C.c_float), ("a", C.c_float), ("n", C.c_float),
                ("seed", C.c_uint32)]


CONST, CURV, NOISE = 1, 2, 4


def build():
    """Compile liboracle.so from its sources (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _lib.fo_last_error.restype = C.c_char_p
        _lib.fo_set_threads(1)  # results never depend on it; callers that time may raise it
    return _lib


def set_threads(n):
    """Threads of the oracle's parallel loops: the seven loops the reference runs with OpenMP
    (the speed functor loops of the global and bounded update, the zero-layer update, both
    distance passes, the status-change flush and Polys::march). Results and list orders do not
    depend on it. Returns the count in effect."""
    return int(lib().fo_set_threads(int(n)))


def _chk(rc):
    if rc != 0:
        raise OracleError(rc, lib().fo_last_error().decode())


def _ivec(v):
    return (C.c_int * len(v))(*[int(x) for x in v])


def _fetch_list(fn, *args):
    n = C.c_size_t(0)
    cap = 256
    while True:
        buf = (C.c_uint32 * cap)()
        _chk(fn(*args, buf, C.c_size_t(cap), C.byref(n)))
        if n.value <= cap:
            return list(buf[: n.value])
        cap = n.value


class Surface:
    """Oracle Surface<D,L>(size, part) with the same call surface as felt_b200.Surface.

    fp64=True runs the same method with distances in double precision (the reference hard-wires
    float, include/Felt/Impl/Common.hpp:40): the run error figures are taken against."""

    def __init__(self, size, part, layers, fp64=False):
        self.D = len(size)
        self.L = layers
        self.size = tuple(int(s) for s in size)
        self.part = tuple(int(p) for p in part)
        self.fp64 = bool(fp64)
        h = C.c_void_p()
        make = lib().fo_surface_create64 if fp64 else lib().fo_surface_create
        _chk(make(self.D, self.L, _ivec(size), _ivec(part), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.fo_surface_destroy(h)
            self._h = None

    @staticmethod
    def layer_idx(layer_id, L):
        return layer_id + L

    def seed(self, pos):
        _chk(lib().fo_seed(self._h, _ivec(pos)))

    def update(self, c=None, a=None, n=None, seed=0):
        kind = 0
        if a is not None:
            kind |= CURV
        if n is not None:
            kind |= NOISE
        if c is not None:
            kind |= CONST
        sp = Speed(kind, float(c or 0.0), float(a or 0.0), float(n or 0.0), int(seed))
        _chk(lib().fo_update_builtin(self._h, C.byref(sp)))

    def update_bounded(self, lo, hi, c=None, a=None, n=None, seed=0):
        kind = (CURV if a is not None else 0) | (NOISE if n is not None else 0) | (
            CONST if c is not None else 0)
        sp = Speed(kind, float(c or 0.0), float(a or 0.0), float(n or 0.0), int(seed))
        _chk(lib().fo_update_bounded(self._h, _ivec(lo), _ivec(hi), C.byref(sp)))

    def update_start(self):
        _chk(lib().fo_update_start(self._h))

    def delta(self, pos, val):
        _chk(lib().fo_delta(self._h, _ivec(pos), C.c_float(val)))

    def update_end(self):
        _chk(lib().fo_update_end(self._h))

    def snapshot(self):
        n = int(np.prod(self.size))
        out = np.zeros(n, dtype=np.float32)
        _chk(lib().fo_snapshot(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(n)))
        return out.reshape(self.size)

    def snapshot64(self):
        """The dense snapshot in the surface's own arithmetic, as float64."""
        n = int(np.prod(self.size))
        out = np.zeros(n, dtype=np.float64)
        _chk(lib().fo_snapshot64(self._h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                 C.c_size_t(n)))
        return out.reshape(self.size)

    def get(self, pos):
        v = C.c_float()
        _chk(lib().fo_get(self._h, _ivec(pos), C.byref(v)))
        return v.value

    def curv(self, pos):
        v = C.c_float()
        _chk(lib().fo_curv(self._h, _ivec(pos), C.byref(v)))
        return v.value

    def numeric(self, pos):
        """grad, gradF, gradB, gradC, gradE (D values each) and divergence at a node."""
        out = (C.c_float * (5 * self.D + 1))()
        _chk(lib().fo_numeric(self._h, _ivec(pos), out))
        return np.array(out, dtype=np.float32)

    def numeric_f(self, pos):
        """The Numeric API at a real position: grad, gradF, gradB, gradC, gradE (D values
        each), divergence, curv and the interpolated value."""
        p = (C.c_float * self.D)(*[float(np.float32(x)) for x in pos])
        out = (C.c_float * (5 * self.D + 3))()
        _chk(lib().fo_numeric_f(self._h, p, out))
        return np.array(out, dtype=np.float32)

    def save(self):
        """Surface::save: the surface file (the reference's cereal binary layout) as bytes."""
        n = C.c_size_t()
        _chk(lib().fo_save(self._h, None, C.c_size_t(0), C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        _chk(lib().fo_save(self._h, buf, C.c_size_t(n.value), C.byref(n)))
        return bytes(buf)

    @classmethod
    def load(cls, data):
        """Surface::load: a new surface from a surface file."""
        h = C.c_void_p()
        raw = (C.c_uint8 * len(data)).from_buffer_copy(data)
        _chk(lib().fo_load(raw, C.c_size_t(len(data)), C.byref(h)))
        obj = cls.__new__(cls)
        obj._h = h
        d, l_ = C.c_int(), C.c_int()
        sz, pt = (C.c_int * 3)(), (C.c_int * 3)()
        _chk(lib().fo_info(h, C.byref(d), C.byref(l_), sz, pt))
        obj.D, obj.L = d.value, l_.value
        obj.size = tuple(sz[: obj.D])
        obj.part = tuple(pt[: obj.D])
        return obj

    def rays(self, origins, dirs):
        """Surface::ray for each (origin, direction) row; rows of FLT_MAX where missed."""
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, self.D)
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, self.D)
        out = np.zeros_like(o)
        _chk(lib().fo_ray(self._h, o.ctypes.data_as(C.POINTER(C.c_float)),
                          d.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(o.shape[0]),
                          out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def ray(self, origin, direction):
        return self.rays([origin], [direction])[0]

    def partitions(self):
        cnt = C.c_size_t()
        cs = (C.c_int * self.D)()
        co = (C.c_int * self.D)()
        _chk(lib().fo_partitions(self._h, C.byref(cnt), cs, co))
        return cnt.value, tuple(cs), tuple(co)

    def layer_list(self, part, layer_idx):
        return _fetch_list(lib().fo_layer_list, self._h, C.c_size_t(part), C.c_int(layer_idx))

    def partition_list(self, layer_idx, which=0):
        return _fetch_list(lib().fo_partition_list, self._h, C.c_int(which), C.c_int(layer_idx))

    def delta_partitions(self, layer_idx):
        return self.partition_list(layer_idx, which=1)

    def status_partitions(self, layer_idx):
        return self.partition_list(layer_idx, which=2)

    def affected_partitions(self, layer_idx):
        return self.partition_list(layer_idx, which=3)

    def affected_list(self, part, layer_idx):
        return _fetch_list(lib().fo_affected_list, self._h, C.c_size_t(part), C.c_int(layer_idx))

    def partition_state(self, part):
        a = C.c_int()
        bg = C.c_float()
        _chk(lib().fo_partition_state(self._h, C.c_size_t(part), C.byref(a), C.byref(bg)))
        return bool(a.value), bg.value

    def stats(self):
        a = C.c_size_t()
        b = C.c_size_t()
        _chk(lib().fo_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def band_size(self):
        n = C.c_size_t()
        _chk(lib().fo_band_size(self._h, C.byref(n)))
        return n.value

    def layer_size(self, layer_id):
        """Total nodes in a layer over all partitions (test_Surface.cpp:1711-1727)."""
        li = layer_id + self.L
        return sum(len(self.layer_list(p, li)) for p in self.partition_list(li))

    def dump(self):
        return np.array(_fetch_list(lib().fo_dump, self._h), dtype=np.uint32)

    def run_steps(self, steps, c=None, a=None, n=None, seed=0):
        kind = (CURV if a is not None else 0) | (NOISE if n is not None else 0) | (
            CONST if c is not None else 0)
        sp = Speed(kind, float(c or 0.0), float(a or 0.0), float(n or 0.0), int(seed))
        nu = C.c_double()
        secs = C.c_double()
        _chk(lib().fo_run_steps(self._h, C.byref(sp), C.c_int(steps), C.byref(nu),
                                C.byref(secs)))
        return nu.value, secs.value


class Polys:
    def __init__(self, surface: Surface):
        self.surface = surface
        h = C.c_void_p()
        _chk(lib().fo_polys_create(surface._h, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.fo_polys_destroy(h)
            self._h = None

    def notify(self):
        _chk(lib().fo_polys_notify(self._h))

    def march(self):
        _chk(lib().fo_polys_march(self._h))

    def invalidate(self):
        _chk(lib().fo_polys_invalidate(self._h))

    def march_partition(self, part):
        _chk(lib().fo_polys_march_partition(self._h, C.c_size_t(part)))

    def changes(self):
        return _fetch_list(lib().fo_polys_changes, self._h)

    def partition(self, part):
        D = self.surface.D
        per = 2 * D if D == 3 else D
        nv = C.c_size_t()
        ns = C.c_size_t()
        act = C.c_int()
        _chk(lib().fo_polys_partition(self._h, C.c_size_t(part), None, C.c_size_t(0), None,
                                      C.c_size_t(0), C.byref(nv), C.byref(ns), C.byref(act)))
        vtx = np.zeros(max(1, nv.value * per), dtype=np.float32)
        spx = np.zeros(max(1, ns.value * D), dtype=np.uint32)
        _chk(lib().fo_polys_partition(self._h, C.c_size_t(part),
                                      vtx.ctypes.data_as(C.POINTER(C.c_float)),
                                      C.c_size_t(vtx.size),
                                      spx.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      C.c_size_t(spx.size), C.byref(nv), C.byref(ns),
                                      C.byref(act)))
        return (vtx[: nv.value * per].reshape(nv.value, per), spx[: ns.value * D].reshape(
            ns.value, D), bool(act.value))

    def partition64(self, part):
        """partition()'s vertices in the surface's own arithmetic, as float64 rows."""
        D = self.surface.D
        per = 2 * D if D == 3 else D
        nv = C.c_size_t()
        _chk(lib().fo_polys_partition64(self._h, C.c_size_t(part), None, C.c_size_t(0),
                                        C.byref(nv)))
        vtx = np.zeros(max(1, nv.value * per), dtype=np.float64)
        _chk(lib().fo_polys_partition64(self._h, C.c_size_t(part),
                                        vtx.ctypes.data_as(C.POINTER(C.c_double)),
                                        C.c_size_t(vtx.size), C.byref(nv)))
        return vtx[: nv.value * per].reshape(nv.value, per)

    def totals(self):
        nv = C.c_size_t()
        ns = C.c_size_t()
        _chk(lib().fo_polys_totals(self._h, C.byref(nv), C.byref(ns)))
        return nv.value, ns.value


FLT_EPS = float(np.finfo(np.float32).eps)


def layer_ids(phi):
    """Surface::layer_id of every value (Surface.hpp:1694-1697): round(v + FLT_EPSILON), halves
    away from zero."""
    x = np.asarray(phi, dtype=np.float64) + FLT_EPS
    return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)


def fp64_errors(snap32, snap64, L, polys=()):
    """Error of an FP32 result against the FP64 run of the same method.

    phi: max |phi32 - phi64| over the nodes whose layer is the same in both runs and inside the
    band (|layer| <= L), with the count of such nodes and of nodes whose layer differs.
    vertices: polys yields (vtx32, spx32, vtx64, spx64) per partition; over the partitions with
    identical simplices (same topology) the max difference of positions and, in 3D, of normals."""
    a = np.asarray(snap32, dtype=np.float64)
    b = np.asarray(snap64, dtype=np.float64)
    la, lb = layer_ids(a), layer_ids(b)
    band = (np.abs(la) <= L) | (np.abs(lb) <= L)
    same = band & (la == lb)
    out = {"phi_max_abs": float(np.abs(a - b)[same].max()) if same.any() else 0.0,
           "phi_nodes": int(same.sum()), "layer_differs": int((band & (la != lb)).sum())}
    vmax = nmax = 0.0
    nparts = ndiff = 0
    for v32, s32, v64, s64 in polys:
        if s32.shape != s64.shape or not np.array_equal(s32, s64) or v32.shape != v64.shape:
            ndiff += 1
            continue
        nparts += 1
        if v32.size:
            d = np.abs(np.asarray(v32, dtype=np.float64) - v64)
            D = s32.shape[1] if s32.ndim == 2 and s32.shape[1] else (v32.shape[1] // 2)
            vmax = max(vmax, float(d[:, :D].max()))
            if v32.shape[1] > D:
                nmax = max(nmax, float(d[:, D:].max()))
    out.update({"vertex_max_abs": vmax, "normal_max_abs": nmax, "poly_partitions": nparts,
                "poly_topology_differs": ndiff})
    return out
