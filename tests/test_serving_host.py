"""Host-side logic of the serving path (no GPU): the request stream is deterministic and has the
configured distribution, and the server's admission bound (fg_request_bricks, host arithmetic
in the C ABI) grows with a request's reach and its speed and stops at the grid."""
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


def _bricks(size, steps, speed, L=2, part=(8, 8, 8)):
    from felt_b200.serving import Request, reserve_bricks
    return reserve_bricks(Request(size, (0,) * len(size), speed, steps, False), L, part)


def test_reservation_bounds():
    small = _bricks((128, 128, 128), 4, dict(c=-0.5))
    big = _bricks((128, 128, 128), 60, dict(c=-0.5))
    assert small < big
    # a 4-step request reaches L + 2 + 4 = 8 cells: a 17-cell span, at most 4 partitions per axis
    assert small == 4 ** 3
    # never more bricks than the grid has partitions (a partial one adds one per axis)
    huge = _bricks((64, 64, 64), 64, dict(a=-0.3, c=-0.2))
    assert huge <= (64 // 8 + 1) ** 3
    # a speed that can exceed one cell per step reaches further
    slow = _bricks((256, 256, 256), 10, dict(c=-0.5))
    fast = _bricks((256, 256, 256), 10, dict(c=-3.0))
    assert fast > slow
    # curvature counts with its largest magnitude (D): 0.5 * 3 + 0.2 > 1
    curv = _bricks((256, 256, 256), 10, dict(a=-0.5, c=-0.2))
    assert curv > slow
    # reach 2 + 2 + 5 = 9 cells: a 19-cell span, at most 3 partitions of 16 per axis
    assert _bricks((512, 512), 5, dict(c=-0.4), part=(16, 16)) == 3 ** 2


def test_brick_bytes():
    from felt_b200.serving import brick_bytes
    # per leaf phi, delta, lookup, 5 lists, status, 5 status lists, 2 affected lookups,
    # 2 x 5 affected lists, claim, claimed-leaf list; per brick the list counts and queues
    assert brick_bytes(2, (8, 8, 8)) == 512 * 65 + 4 * 27
    assert math.isclose(brick_bytes(3, (16, 16, 16)),
                        4096 * (4 + 4 + 2 + 14 + 1 + 14 + 4 + 28 + 8 + 2) + 4 * 35)
