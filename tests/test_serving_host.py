"""Host-side logic of the serving path (no GPU): the request stream is deterministic and has the
configured distribution, and the admission reservation bounds grow with a request's reach and
stop at the grid."""
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_request_stream_is_seeded_and_in_range():
    import bench
    cfg = bench.CONFIGS["c5"]
    a = bench.serve_requests(cfg, 1000)
    b = bench.serve_requests(cfg, 1000)
    assert [(t, r.size, r.centre, r.steps, r.polys, r.kind) for t, r in a] == \
           [(t, r.size, r.centre, r.steps, r.polys, r.kind) for t, r in b]
    assert len(a) == min(cfg["max_requests"], int(1000 * cfg["max_seconds"]))
    times = [t for t, _ in a]
    assert all(x < y for x, y in zip(times, times[1:]))
    mean_gap = times[-1] / len(times)
    assert 0.8e-3 < mean_gap < 1.2e-3
    for _, r in a:
        e = r.size[0]
        assert 32 <= e <= 256 and r.size == (e, e, e)
        assert 1 <= r.steps <= 64
        lo, hi = -e // 2 + 3, e // 2 - 4
        assert all(lo <= c <= hi for c in r.centre)
    kinds = {r.kind for _, r in a}
    assert kinds == {"constant", "curvature", "noise"}


def test_reservation_bounds():
    from felt_b200.serving import Request, brick_bytes, reserve_bytes
    part = (8, 8, 8)
    small = Request((128, 128, 128), (0, 0, 0), dict(c=-0.5), 4, False, "constant")
    big = Request((128, 128, 128), (0, 0, 0), dict(c=-0.5), 60, False, "constant")
    nb_s, by_s = reserve_bytes(small, 2, part)
    nb_b, by_b = reserve_bytes(big, 2, part)
    assert nb_s < nb_b and by_s < by_b
    # never more bricks than the grid has partitions
    huge = Request((64, 64, 64), (0, 0, 0), dict(c=-0.5), 64, False, "curvature")
    nb_h, _ = reserve_bytes(huge, 2, part)
    assert nb_h <= (math.ceil(64 / 8) + 1) ** 3
    assert brick_bytes(2, part) == 512 * 63 + 4 * 21
