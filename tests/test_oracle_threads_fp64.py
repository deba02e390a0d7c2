"""The oracle itself: its threaded loops (the seven loops the reference runs with OpenMP) give
the same lists, orders, values and polygons as one thread, and its FP64 run of the same method
stays within a few float ulps of the FP32 run with the same layer membership."""
import numpy as np

from oracle import oracle as O

CASES = [
    # D, L, size, part, seed, schedule (steps, speed)
    (3, 2, (64, 64, 64), (8, 8, 8), (0, 0, 0),
     [(20, dict(c=-0.5)), (15, dict(a=-0.3, n=0.2, seed=4, c=0.1))]),
    (3, 3, (96, 96, 96), (16, 16, 16), (3, -2, 1),
     [(15, dict(c=-0.8)), (10, dict(a=-0.2, n=0.1, seed=7))]),
    (2, 2, (300, 300), (16, 16), (10, -5), [(30, dict(c=-0.7)), (10, dict(c=0.6))]),
]


def _run(threads, D, L, size, part, seed, schedule, fp64=False):
    O.set_threads(threads)
    try:
        s = O.Surface(size, part, L, fp64=fp64)
        p = O.Polys(s)
        s.seed(seed)
        k = 0
        for n, sp in schedule:
            for _ in range(n):
                s.update(**sp)
                p.notify()
                k += 1
                if k % 5 == 0:
                    p.march()
        # a bounded update (the reference's threaded loop at Surface.hpp:336)
        lo = tuple(c - 6 for c in seed)
        hi = tuple(c + 6 for c in seed)
        s.update_bounded(lo, hi, c=-0.3)
        p.notify()
        p.march()
        parts = [p.partition(pc) for pc in range(s.partitions()[0])]
        return s, p, parts
    finally:
        O.set_threads(1)


def test_threaded_loops_equal_one_thread():
    for case in CASES:
        a, pa, parts_a = _run(1, *case)
        b, pb, parts_b = _run(8, *case)
        assert np.array_equal(a.dump(), b.dump()), case[2]
        assert np.array_equal(a.snapshot(), b.snapshot()), case[2]
        assert pa.changes() == pb.changes()
        for (va, sa, aa), (vb, sb, ab) in zip(parts_a, parts_b):
            assert aa == ab
            assert np.array_equal(sa, sb)
            assert np.array_equal(va, vb)


def test_fp64_run_close_to_fp32():
    for case in CASES:
        D, L = case[0], case[1]
        a, pa, parts_a = _run(4, *case)
        b, pb, _ = _run(4, *case, fp64=True)
        # the same method in double: same lists on these cases, values within a few ulps
        assert np.array_equal(a.dump(), b.dump()), case[2]
        pairs = []
        for pc, (v, sx, _) in enumerate(parts_a):
            pairs.append((v, sx, pb.partition64(pc), pb.partition(pc)[1]))
        errs = O.fp64_errors(a.snapshot(), b.snapshot64(), L, pairs)
        # the figures are the FP32 method's own error: roughly 1e-7..1e-6 for smooth speeds,
        # up to ~1e-3 where curvature of a noise-roughened surface amplifies rounding (vertex
        # positions interpolate between nearly equal values there and move further); the
        # bounds here only catch a broken FP64 run
        assert errs["layer_differs"] == 0
        assert 0 < errs["phi_nodes"]
        assert errs["phi_max_abs"] < 0.05, errs
        assert errs["vertex_max_abs"] < 0.5, errs
        assert errs["poly_topology_differs"] == 0, errs
        # the FP64 values are not just the FP32 ones widened
        assert not np.array_equal(a.snapshot().astype(np.float64), b.snapshot64())


def test_layer_ids_round_half_away():
    # v + FLT_EPSILON, then halves away from zero: -0.5 + eps rounds to 0, 1.5 - 2e-7 + eps to 1
    v = np.array([0.5, -0.5, 1.5 - 2e-7, -2.4999, 2.5, 0.0, -1e-9, -1.5], dtype=np.float64)
    assert [int(x) for x in O.layer_ids(v)] == [1, 0, 1, -2, 3, 0, 0, -1]
