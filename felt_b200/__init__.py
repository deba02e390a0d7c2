"""felt_b200: B200-native sparse-field level sets with the Felt Surface<D,L> / Polys API.

Python binding over the C ABI of libfelt_gpu.so (include/felt_gpu.h). The classes mirror the
reference's C++ API (include/Felt/Surface.hpp, include/Felt/Polys.hpp): Surface(size, part, L)
with seed / update / update_start / delta / update_end / snapshot and the list accessors, and
Polys(surface) with notify / march / invalidate / changes.

All compute runs in the CUDA kernels of libfelt_gpu.so; there is no CPU fallback. If the library
is missing or no CUDA device is present, constructing a Surface raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfelt_gpu.so")
_lib = None

SPEED_CONST, SPEED_CURV, SPEED_NOISE = 1, 2, 4

# Surface::ray_miss (include/Felt/Surface.hpp:62-64): FLT_MAX in every component.
RAY_MISS = float(np.finfo(np.float32).max)


class FeltError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"felt_gpu error {code}: {msg}")
        self.code = code


class Speed(C.Structure):
    _fields_ = [("kind", C.c_int), ("c", C.c_float), ("a", C.c_float), ("n", C.c_float),
                ("seed", C.c_uint32)]


class Config(C.Structure):
    _fields_ = [("brick_capacity", C.c_size_t), ("vertex_capacity", C.c_size_t),
                ("launch_mode", C.c_int), ("dist_split", C.c_int), ("record_passes", C.c_int),
                ("autotune", C.c_int), ("delta_kernel", C.c_int), ("fuse_passes", C.c_int),
                ("reserved", C.c_int * 2)]


def make_config(brick_capacity=0, vertex_capacity=0, launch_mode=0, dist_split=0,
                record_passes=0, autotune=False, delta_kernel=0, fuse_passes=0):
    """fg_config: pool sizes and launch tuning (launch_mode 0 automatic, 1 the whole global
    update as one CUDA graph, 2 every kernel launched from the host, no graphs; dist_split warps per partition
    entry in the first distance pass; record_passes 1 warp / 2 block per entry in the
    recording passes; delta_kernel of curvature speeds 1 direct / 2 staged brick + halo;
    fuse_passes 1 separate / 2 fused / 3 tiled (per brick in shared memory) distance passes;
    0 = automatic everywhere; autotune: dist_split and record_passes left at 0 take the values
    autotune() measures)."""
    return Config(int(brick_capacity), int(vertex_capacity), int(launch_mode), int(dist_split),
                  int(record_passes), 1 if autotune else 0, int(delta_kernel),
                  int(fuse_passes))


def autotune_candidates(part):
    """The (dist_split, record_passes) pairs the tuner times for a partition shape."""
    buf = (C.c_int * 32)()
    n = C.c_size_t()
    _chk(lib().fg_autotune_candidates(len(part), _ivec(part), buf, C.c_size_t(32), C.byref(n)))
    return [(buf[2 * i], buf[2 * i + 1]) for i in range(n.value)]


def autotune(part, layers, force=False):
    """fg_autotune: the fastest (dist_split, record_passes) for this partition shape and layer
    count on the current device, timed on a scratch surface (or cached); with each candidate's
    device ms per update when it was timed."""
    cfg = make_config()
    ms = (C.c_double * 32)()
    n = C.c_size_t()
    _chk(lib().fg_autotune(len(part), int(layers), _ivec(part), 1 if force else 0, C.byref(cfg),
                           ms, C.c_size_t(32), C.byref(n)))
    return dict(dist_split=cfg.dist_split, record_passes=cfg.record_passes,
                ms=dict(zip(autotune_candidates(part), list(ms)[:n.value])))


def _tuning(fn, h):
    out = (C.c_int * 8)()
    _chk(fn(h, out))
    return dict(launch_mode=out[0], dist_split=out[1], record_passes=out[2],
                delta_kernel=out[3], fuse_passes=out[4])


def build():
    """Compile libfelt_gpu.so for sm_100a (nvcc; no GPU needed)."""
    subprocess.run(["bash", os.path.join(_HERE, "csrc", "build.sh")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FeltError(-2, f"{LIB_PATH} is not built; run felt_b200.build()")
        _lib = C.CDLL(LIB_PATH)
        _lib.fg_last_error.restype = C.c_char_p
    return _lib


def _chk(rc):
    if rc != 0:
        raise FeltError(rc, lib().fg_last_error().decode())


def _ivec(v):
    return (C.c_int * len(v))(*[int(x) for x in v])


def _fetch(fn, *args):
    n = C.c_size_t(0)
    cap = 256
    while True:
        buf = (C.c_uint32 * cap)()
        _chk(fn(*args, buf, C.c_size_t(cap), C.byref(n)))
        if n.value <= cap:
            return list(buf[: n.value])
        cap = n.value


QUERY = {"get": 0, "curv": 1, "divergence": 2, "inside": 3, "grad": 4, "gradF": 5, "gradB": 6,
         "gradC": 7, "gradE": 8}


def _query(fn_real, fn_nodes, head, D, what, pos):
    """Runs fg_query (float positions) or fg_query_nodes (integer positions) and shapes the
    result: (n,) for scalar queries, (n, D) for the gradients."""
    code = QUERY[what] if isinstance(what, str) else int(what)
    p = np.asarray(pos)
    if p.ndim == 1:
        p = p[None, :]
    if p.ndim != 2 or p.shape[1] != D:
        raise ValueError("positions must be (n, %d)" % D)
    w = D if code >= QUERY["grad"] else 1
    out = np.empty((p.shape[0], w), dtype=np.float32)
    optr = out.ctypes.data_as(C.POINTER(C.c_float))
    n = C.c_size_t(p.shape[0])
    if np.issubdtype(p.dtype, np.integer):
        a = np.ascontiguousarray(p, dtype=np.int32)
        _chk(fn_nodes(*head, C.c_int(code), a.ctypes.data_as(C.POINTER(C.c_int)), n, optr))
    else:
        a = np.ascontiguousarray(p, dtype=np.float32)
        _chk(fn_real(*head, C.c_int(code), a.ctypes.data_as(C.POINTER(C.c_float)), n, optr))
    return out if w > 1 else out[:, 0]


def _ray_arrays(origins, dirs, D):
    o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, D)
    d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, D)
    if o.shape != d.shape:
        raise ValueError(f"origins {o.shape} and dirs {d.shape} differ")
    return o, d


def launch_count():
    """Kernels launched by libfelt_gpu.so in this process."""
    n = C.c_longlong()
    _chk(lib().fg_launch_count(C.byref(n)))
    return n.value


def profile_enable(on=True):
    """Bracket every library kernel launch with CUDA events (per-kernel device time)."""
    _chk(lib().fg_profile_enable(1 if on else 0))


def profile_reset():
    _chk(lib().fg_profile_reset())


def profile_only(kernel=None):
    """Bracket only the launches of one kernel while profiling (None = every kernel)."""
    _chk(lib().fg_profile_only(kernel.encode() if kernel else None))


def profile_read():
    """{kernel name: (total ms, launches)} accumulated while profiling was enabled."""
    n = C.c_size_t()
    _chk(lib().fg_profile_count(C.byref(n)))
    out = {}
    name = C.create_string_buffer(128)
    for i in range(n.value):
        ms = C.c_double()
        k = C.c_longlong()
        _chk(lib().fg_profile_entry(C.c_size_t(i), name, C.c_size_t(128), C.byref(ms),
                                    C.byref(k)))
        out[name.value.decode()] = (ms.value, k.value)
    return out


def make_speed(c=None, a=None, n=None, seed=0):
    """Builtin speed: [a*curv] + [n*noise(pos, seed)] + [c], terms present when given."""
    kind = (SPEED_CURV if a is not None else 0) | (SPEED_NOISE if n is not None else 0) | (
        SPEED_CONST if c is not None else 0)
    return Speed(kind, float(c or 0.0), float(a or 0.0), float(n or 0.0), int(seed))


class Surface:
    """Felt::Surface<D,L>(size, size_partition) on the GPU (include/Felt/Surface.hpp:163-173)."""

    def __init__(self, size, part, layers, brick_capacity=0, vertex_capacity=0, **tuning):
        """tuning: launch_mode, dist_split, record_passes, delta_kernel, autotune (see
        make_config)."""
        self.D = len(size)
        self.L = int(layers)
        self.size = tuple(int(s) for s in size)
        self.part = tuple(int(p) for p in part)
        cfg = make_config(brick_capacity, vertex_capacity, **tuning)
        h = C.c_void_p()
        _chk(lib().fg_surface_create(self.D, self.L, _ivec(size), _ivec(part), C.byref(cfg),
                                     C.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.fg_surface_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def seed(self, pos):
        _chk(lib().fg_seed(self._h, _ivec(pos)))

    def update(self, c=None, a=None, n=None, seed=0):
        sp = make_speed(c, a, n, seed)
        _chk(lib().fg_update_builtin(self._h, C.byref(sp)))

    def update_bounded(self, lo, hi, c=None, a=None, n=None, seed=0):
        sp = make_speed(c, a, n, seed)
        _chk(lib().fg_update_bounded(self._h, _ivec(lo), _ivec(hi), C.byref(sp)))

    def update_start(self):
        _chk(lib().fg_update_start(self._h))

    def delta(self, pos, val):
        _chk(lib().fg_delta(self._h, _ivec(pos), C.c_float(val)))

    def update_end(self):
        _chk(lib().fg_update_end(self._h))

    def tuning(self):
        """The launch tuning in effect (fg_surface_tuning)."""
        return _tuning(lib().fg_surface_tuning, self._h)

    def snapshot(self):
        n = int(np.prod(self.size))
        out = np.zeros(n, dtype=np.float32)
        _chk(lib().fg_snapshot(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(n),
                               0))
        return out.reshape(self.size)

    def snapshot_into(self, dev_ptr, n):
        """Snapshot into device memory (e.g. a torch CUDA tensor's data_ptr())."""
        _chk(lib().fg_snapshot(self._h, C.c_void_p(dev_ptr), C.c_size_t(n), 1))

    def get(self, pos):
        v = C.c_float()
        _chk(lib().fg_get(self._h, _ivec(pos), C.byref(v)))
        return v.value

    def save(self):
        """Surface::save (include/Felt/Surface.hpp:180-183): the surface file, in the reference's
        format, as bytes."""
        n = C.c_size_t()
        _chk(lib().fg_save(self._h, None, C.c_size_t(0), C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        _chk(lib().fg_save(self._h, buf, C.c_size_t(n.value), C.byref(n)))
        return bytes(buf)

    @classmethod
    def load(cls, data, brick_capacity=0, vertex_capacity=0, **tuning):
        """Surface::load (include/Felt/Surface.hpp:185-196): a new surface from a surface file
        (bytes); dimensions, layers and sizes come from the file."""
        raw = (C.c_uint8 * len(data)).from_buffer_copy(data)
        cfg = make_config(brick_capacity, vertex_capacity, **tuning)
        h = C.c_void_p()
        _chk(lib().fg_load(raw, C.c_size_t(len(data)), C.byref(cfg), C.byref(h)))
        obj = cls.__new__(cls)
        obj._h = h
        d, l_ = C.c_int(), C.c_int()
        cnt = C.c_size_t()
        cs, co = (C.c_int * 3)(), (C.c_int * 3)()
        _chk(lib().fg_surface_info(h, C.byref(d), C.byref(l_), cs, co))
        obj.D, obj.L = d.value, l_.value
        obj.size = tuple(cs[: obj.D])
        obj.part = tuple(co[: obj.D])
        return obj

    def rays(self, origins, dirs):
        """Surface::ray (include/Felt/Surface.hpp:468-616) for each (origin, direction) row: the
        point where the ray meets the zero curve, or a row of RAY_MISS where it misses."""
        o, d = _ray_arrays(origins, dirs, self.D)
        out = np.empty_like(o)
        _chk(lib().fg_ray(self._h, o.ctypes.data_as(C.POINTER(C.c_float)),
                          d.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(o.shape[0]),
                          out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def query(self, what, positions):
        """The isogrid's Numeric API at n positions: what is one of QUERY's names ("get",
        "curv", "divergence", "inside", "grad", "gradF", "gradB", "gradC", "gradE"); integer
        positions are nodes, float positions real positions (get = interp there)."""
        return _query(lib().fg_query, lib().fg_query_nodes, (self._h,), self.D, what, positions)

    def ray(self, origin, direction):
        """Surface::ray(origin, dir) for one ray."""
        return self.rays([origin], [direction])[0]

    def rays_device(self, origins_ptr, dirs_ptr, n, hits_ptr, order_mode=0):
        """rays() over device arrays of n*D floats (e.g. torch CUDA tensors' data_ptr()).
        order_mode: 0 (default) merges per-axis candidate lists, 1 finds each next candidate by
        a full walk, 2 merges per-axis cursors; same order and hits, 1 and 2 are slower."""
        _chk(lib().fg_ray_device(self._h, C.c_void_p(origins_ptr), C.c_void_p(dirs_ptr),
                                 C.c_size_t(n), C.c_void_p(hits_ptr), C.c_int(int(order_mode))))

    def partitions(self):
        cnt = C.c_size_t()
        cs = (C.c_int * self.D)()
        co = (C.c_int * self.D)()
        _chk(lib().fg_partitions(self._h, C.byref(cnt), cs, co))
        return cnt.value, tuple(cs), tuple(co)

    def layer_list(self, part, layer_idx):
        return _fetch(lib().fg_layer_list, self._h, C.c_size_t(part), C.c_int(layer_idx))

    def partition_list(self, layer_idx):
        return _fetch(lib().fg_partition_list, self._h, C.c_int(layer_idx))

    def delta_partitions(self, layer_idx):
        return _fetch(lib().fg_delta_partitions, self._h, C.c_int(layer_idx))

    def status_partitions(self, layer_idx):
        return _fetch(lib().fg_status_partitions, self._h, C.c_int(layer_idx))

    def affected_partitions(self, layer_idx):
        return _fetch(lib().fg_affected_partitions, self._h, C.c_int(layer_idx))

    def affected_list(self, part, layer_idx):
        return _fetch(lib().fg_affected_list, self._h, C.c_size_t(part), C.c_int(layer_idx))

    def partition_state(self, part):
        a = C.c_int()
        bg = C.c_float()
        _chk(lib().fg_partition_state(self._h, C.c_size_t(part), C.byref(a), C.byref(bg)))
        return bool(a.value), bg.value

    def stats(self):
        a = C.c_size_t()
        b = C.c_size_t()
        _chk(lib().fg_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def band_size(self):
        n = C.c_size_t()
        _chk(lib().fg_band_size(self._h, C.byref(n)))
        return n.value

    def iterations(self):
        """Convergence-loop iterations of the last update (fg_update_iterations)."""
        n = C.c_int()
        _chk(lib().fg_update_iterations(self._h, C.byref(n)))
        return n.value

    def work_units(self):
        """(distance-pass nodes, zero-layer nodes, flush edits, marched cells) so far."""
        out = (C.c_ulonglong * 8)()
        _chk(lib().fg_work_units(self._h, out, C.c_size_t(8)))
        return tuple(out[:4])

    def stream(self):
        """cudaStream_t (as int) that all work of this surface runs on."""
        p = C.c_void_p()
        _chk(lib().fg_surface_stream(self._h, C.byref(p)))
        return p.value or 0

    def node_updates(self):
        """Band nodes processed by all global updates so far (band size at each start)."""
        n = C.c_ulonglong()
        _chk(lib().fg_node_updates(self._h, C.byref(n)))
        return n.value

    def layer_size(self, layer_id):
        li = layer_id + self.L
        return sum(len(self.layer_list(p, li)) for p in self.partition_list(li))

    def dump(self):
        return np.array(_fetch(lib().fg_dump, self._h), dtype=np.uint32)


class Batch:
    """Many independent Surface<D,L> (same D, L, partition shape; any grid sizes) advanced by the
    same kernel launches. Per surface the results equal a separate Surface's."""

    def __init__(self, sizes, part, layers, brick_capacity=0, vertex_capacity=0, **tuning):
        """tuning: launch_mode, dist_split, record_passes, delta_kernel, autotune (see
        make_config)."""
        self.n = len(sizes)
        self.D = len(part)
        self.L = int(layers)
        self.part = tuple(int(p) for p in part)
        self.sizes = [tuple(int(x) for x in s) for s in sizes]
        flat = [x for s in self.sizes for x in s]
        cfg = make_config(brick_capacity, vertex_capacity, **tuning)
        h = C.c_void_p()
        _chk(lib().fg_batch_create(self.D, self.L, _ivec(part), C.c_size_t(self.n), _ivec(flat),
                                   C.byref(cfg), C.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.fg_batch_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def seed(self, centres):
        flat = [int(x) for c in centres for x in c]
        _chk(lib().fg_batch_seed(self._h, _ivec(flat)))

    def speed_array(self, speeds):
        """The per-surface speeds as the C array update() passes down (build it once when the
        speeds do not change from step to step)."""
        if isinstance(speeds, dict):
            speeds = [speeds] * self.n
        if len(speeds) != self.n:
            raise ValueError("one speed per surface")
        return (Speed * self.n)(*[make_speed(**s) for s in speeds])

    def update(self, speeds):
        """speeds: one dict(c=, a=, n=, seed=) per surface, one dict for all, or an array from
        speed_array()."""
        arr = speeds if isinstance(speeds, C.Array) else self.speed_array(speeds)
        _chk(lib().fg_batch_update(self._h, arr))

    def polys_notify(self):
        _chk(lib().fg_batch_polys_notify(self._h))

    def polys_march(self):
        _chk(lib().fg_batch_polys_march(self._h))

    def polys_invalidate(self):
        _chk(lib().fg_batch_polys_invalidate(self._h))

    def snapshot(self, i):
        n = int(np.prod(self.sizes[i]))
        out = np.zeros(n, dtype=np.float32)
        _chk(lib().fg_batch_snapshot(self._h, C.c_size_t(i),
                                     out.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(n)))
        return out.reshape(self.sizes[i])

    def rays(self, i, origins, dirs):
        """Surface::ray of surface i for each (origin, direction) row (RAY_MISS rows on a miss)."""
        o, d = _ray_arrays(origins, dirs, self.D)
        out = np.empty_like(o)
        _chk(lib().fg_batch_ray(self._h, C.c_size_t(i), o.ctypes.data_as(C.POINTER(C.c_float)),
                                d.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(o.shape[0]),
                                out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def query(self, i, what, positions):
        """Surface.query on surface i."""
        return _query(lib().fg_batch_query, lib().fg_batch_query_nodes,
                      (self._h, C.c_size_t(i)), self.D, what, positions)

    def save(self, i):
        """Surface::save of surface i: the surface file as bytes."""
        n = C.c_size_t()
        _chk(lib().fg_batch_save(self._h, C.c_size_t(i), None, C.c_size_t(0), C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        _chk(lib().fg_batch_save(self._h, C.c_size_t(i), buf, C.c_size_t(n.value), C.byref(n)))
        return bytes(buf)

    def restore(self, i, data):
        """Surface::load of a surface file into surface i, which must be empty."""
        raw = (C.c_uint8 * len(data)).from_buffer_copy(data)
        _chk(lib().fg_batch_restore(self._h, C.c_size_t(i), raw, C.c_size_t(len(data))))

    def dump(self, i):
        return np.array(_fetch(lib().fg_batch_dump, self._h, C.c_size_t(i)), dtype=np.uint32)

    def polys_changes(self, i):
        return _fetch(lib().fg_batch_polys_changes, self._h, C.c_size_t(i))

    def polys_partition(self, i, part):
        D = self.D
        per = 2 * D if D == 3 else D
        nv = C.c_size_t()
        ns = C.c_size_t()
        act = C.c_int()
        _chk(lib().fg_batch_polys_partition(self._h, C.c_size_t(i), C.c_size_t(part), None,
                                            C.c_size_t(0), None, C.c_size_t(0), C.byref(nv),
                                            C.byref(ns), C.byref(act)))
        vtx = np.zeros(max(1, nv.value * per), dtype=np.float32)
        spx = np.zeros(max(1, ns.value * D), dtype=np.uint32)
        _chk(lib().fg_batch_polys_partition(self._h, C.c_size_t(i), C.c_size_t(part),
                                            vtx.ctypes.data_as(C.POINTER(C.c_float)),
                                            C.c_size_t(vtx.size),
                                            spx.ctypes.data_as(C.POINTER(C.c_uint32)),
                                            C.c_size_t(spx.size), C.byref(nv), C.byref(ns),
                                            C.byref(act)))
        return (vtx[: nv.value * per].reshape(nv.value, per),
                spx[: ns.value * D].reshape(ns.value, D), bool(act.value))

    def polys_totals(self):
        nv = C.c_size_t()
        ns = C.c_size_t()
        _chk(lib().fg_batch_polys_totals(self._h, C.byref(nv), C.byref(ns)))
        return nv.value, ns.value

    def node_updates(self):
        n = C.c_ulonglong()
        _chk(lib().fg_batch_node_updates(self._h, C.byref(n)))
        return n.value

    def work_units(self):
        out = (C.c_ulonglong * 8)()
        _chk(lib().fg_batch_work_units(self._h, out, C.c_size_t(8)))
        return tuple(out[:4])

    def stopped(self, i):
        """True once surface i was stopped after an update whose convergence loop did not
        terminate (the reference would loop forever there)."""
        v = C.c_int()
        _chk(lib().fg_batch_surface_stopped(self._h, C.c_size_t(i), C.byref(v)))
        return bool(v.value)

    def pause(self, i, paused=True):
        """Pause (or resume) surface i: later batch calls skip it, leaving it exactly as after
        its own last update."""
        _chk(lib().fg_batch_pause(self._h, C.c_size_t(i), C.c_int(1 if paused else 0)))

    def stream(self):
        p = C.c_void_p()
        _chk(lib().fg_batch_stream(self._h, C.byref(p)))
        return p.value or 0

    def tuning(self):
        """The launch tuning in effect (fg_batch_tuning)."""
        return _tuning(lib().fg_batch_tuning, self._h)


class Polys:
    """Felt::Polys<Surface> (include/Felt/Polys.hpp:1-229) on the GPU."""

    def __init__(self, surface: Surface):
        self.surface = surface
        h = C.c_void_p()
        _chk(lib().fg_polys_create(surface._h, C.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.fg_polys_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def notify(self):
        _chk(lib().fg_polys_notify(self._h))

    def march(self):
        _chk(lib().fg_polys_march(self._h))

    def invalidate(self):
        _chk(lib().fg_polys_invalidate(self._h))

    def march_partition(self, part):
        _chk(lib().fg_polys_march_partition(self._h, C.c_size_t(part)))

    def changes(self):
        return _fetch(lib().fg_polys_changes, self._h)

    def partition(self, part):
        D = self.surface.D
        per = 2 * D if D == 3 else D
        nv = C.c_size_t()
        ns = C.c_size_t()
        act = C.c_int()
        _chk(lib().fg_polys_partition(self._h, C.c_size_t(part), None, C.c_size_t(0), None,
                                      C.c_size_t(0), C.byref(nv), C.byref(ns), C.byref(act)))
        vtx = np.zeros(max(1, nv.value * per), dtype=np.float32)
        spx = np.zeros(max(1, ns.value * D), dtype=np.uint32)
        _chk(lib().fg_polys_partition(self._h, C.c_size_t(part),
                                      vtx.ctypes.data_as(C.POINTER(C.c_float)),
                                      C.c_size_t(vtx.size),
                                      spx.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      C.c_size_t(spx.size), C.byref(nv), C.byref(ns),
                                      C.byref(act)))
        return (vtx[: nv.value * per].reshape(nv.value, per),
                spx[: ns.value * D].reshape(ns.value, D), bool(act.value))

    def totals(self):
        nv = C.c_size_t()
        ns = C.c_size_t()
        _chk(lib().fg_polys_totals(self._h, C.byref(nv), C.byref(ns)))
        return nv.value, ns.value

    def gather(self, parts, vtx_out=None, spx_out=None):
        """Vertices and simplices of several partitions in one call: (vtx, spx, counts).
        vtx_out / spx_out: optional flat float32 / uint32 arrays to copy into (e.g. views of
        pinned host memory kept between calls); they are used when large enough."""
        D = self.surface.D
        per = 2 * D if D == 3 else D
        parts = list(parts)
        arr = (C.c_uint32 * max(1, len(parts)))(*parts)
        counts = np.zeros(2 * max(1, len(parts)), dtype=np.uint32)
        nv = C.c_size_t()
        ns = C.c_size_t()
        _chk(lib().fg_polys_gather(self._h, arr, C.c_size_t(len(parts)), None, C.c_size_t(0),
                                   None, C.c_size_t(0),
                                   counts.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(nv),
                                   C.byref(ns)))
        need_v, need_s = max(1, nv.value * per), max(1, ns.value * D)
        vtx = vtx_out if vtx_out is not None and vtx_out.size >= need_v else np.zeros(
            need_v, dtype=np.float32)
        spx = spx_out if spx_out is not None and spx_out.size >= need_s else np.zeros(
            need_s, dtype=np.uint32)
        _chk(lib().fg_polys_gather(self._h, arr, C.c_size_t(len(parts)),
                                   vtx.ctypes.data_as(C.POINTER(C.c_float)), C.c_size_t(vtx.size),
                                   spx.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_size_t(spx.size),
                                   counts.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(nv),
                                   C.byref(ns)))
        return (vtx[: nv.value * per].reshape(nv.value, per),
                spx[: ns.value * D].reshape(ns.value, D), counts[: 2 * len(parts)].reshape(-1, 2))
