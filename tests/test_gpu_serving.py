"""Serving: a request's result is the same alone as in a mix.

The continuous-batching server (fg_server_* through felt_b200.serving) advances every request in
flight in the same launches; requests submitted while others run take freed slots at the next
step boundary, so a slot's surface is reset and reused many times. Each finished request's
state (lists, orders, values) and polygons must equal the oracle's run of that request alone.
Finished batch surfaces are paused and keep their state."""
import time

import numpy as np
import pytest

from oracle import oracle as O
from tests.dumps import first_difference

pytestmark = pytest.mark.gpu


def _oracle_alone(size, centre, speed, steps, part=(8, 8, 8), L=2):
    o = O.Surface(size, part, L)
    p = O.Polys(o)
    o.seed(centre)
    for _ in range(steps):
        o.update(**speed)
        p.notify()
    p.march()
    return o, p


def test_paused_surfaces_keep_their_state():
    import felt_b200 as fb
    sizes = [(32, 32, 32), (40, 40, 40), (24, 32, 48), (32, 32, 32)]
    centres = [(0, 0, 0), (3, -2, 1), (0, 2, -3), (-2, 0, 1)]
    speeds = [dict(c=-0.4), dict(a=-0.3, c=-0.2), dict(n=0.2, seed=5, c=-0.2), dict(c=-0.6)]
    steps = [3, 9, 6, 9]
    b = fb.Batch(sizes, (8, 8, 8), 2)
    b.seed(centres)
    for k in range(1, max(steps) + 1):
        b.update(speeds)
        b.polys_notify()
        fin = [i for i in range(len(sizes)) if steps[i] == k]
        if fin:
            b.polys_march()
            for i in fin:
                b.pause(i)
    for i in range(len(sizes)):
        o, p = _oracle_alone(sizes[i], centres[i], speeds[i], steps[i])
        d = first_difference(b.dump(i), o.dump())
        assert d is None, f"surface {i}: {d}"
        assert float(np.abs(b.snapshot(i) - o.snapshot()).max()) <= 1e-5
        for part in range(o.partitions()[0]):
            gv, gs, ga = b.polys_partition(i, part)
            ov, os2, oa = p.partition(part)
            assert ga == oa, f"surface {i} partition {part} active"
            assert np.array_equal(gs, os2), f"surface {i} partition {part} simplices"
            if ov.size:
                assert float(np.abs(gv - ov).max()) <= 1e-5


def _requests(n, seed=3):
    from felt_b200.serving import Request
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        e = int(rng.choice([24, 32, 40, 48, 52]))
        kind = ["constant", "curvature", "noise"][k % 3]
        sp = {"constant": dict(c=float(rng.uniform(-0.6, -0.2))),
              "curvature": dict(a=-0.3, c=-0.2),
              "noise": dict(n=0.2, seed=int(rng.integers(0, 1000)), c=-0.2)}[kind]
        c = tuple(int(x) for x in rng.integers(-4, 5, size=3))
        reqs.append(Request((e, e, e), c, sp, int(rng.integers(1, 14)), bool(k % 2), kind,
                            rid=k))
    return reqs


def _check_alone(srv, r, res):
    o, p = _oracle_alone(r.size, r.centre, r.speed, r.steps)
    d = first_difference(res.dump, o.dump())
    assert d is None, f"request {r.rid}: {d}"
    assert res.steps_done == r.steps
    assert res.latency >= 0 and res.done >= res.admitted >= res.arrival - 1e-6
    if r.polys:
        geo = srv.polys(r.rid)
        assert len(geo) == o.partitions()[0]
        nv = ns = 0
        for part, (gv, gs) in enumerate(geo):
            ov, os2, _ = p.partition(part)
            assert np.array_equal(gs, os2), f"request {r.rid} partition {part} simplices"
            if ov.size:
                assert float(np.abs(gv - ov).max()) <= 1e-5
            nv += len(gv)
            ns += len(gs)
        assert (res.vertices, res.simplices) == (nv, ns)


def test_server_results_equal_alone():
    """Three slots, eighteen requests submitted in three bursts while the earlier ones run: each
    slot is reused for several requests of different grid sizes, speeds and step counts."""
    from felt_b200.serving import Server
    reqs = _requests(18)
    srv = Server(slots=3, max_size=(64, 64, 64), brick_capacity=20000, keep_outputs=True)
    try:
        for burst in (reqs[:6], reqs[6:12], reqs[12:]):
            steps0 = srv.stats()["steps"]
            for r in burst:
                r.arrival = srv.now()
                assert srv.submit(r)
            # let the burst get going, so the next one arrives while it runs
            t_end = time.perf_counter() + 5.0
            while srv.stats()["steps"] < steps0 + 3 and time.perf_counter() < t_end:
                time.sleep(0.002)
        assert srv.drain(300)
        res = {r.rid: r for r in srv.results()}
        st = srv.stats()
        assert sorted(res) == list(range(len(reqs)))
        assert st["started"] == len(reqs) and st["completed"] == len(reqs)
        assert st["failed"] == 0
        # requests overlapped: fewer batched steps than the steps of all requests one by one
        assert st["steps"] < sum(r.steps for r in reqs)
        for r in reqs:
            _check_alone(srv, r, res[r.rid])
        assert st["node_updates"] == sum(x.node_updates for x in res.values())
    finally:
        srv.close()


def test_slot_reuse_from_larger_to_smaller_grids():
    """One slot: a 64^3 request, then a 24^3, then a partial-partition 37x50x29 grid: the reset
    leaves nothing of the previous request behind."""
    from felt_b200.serving import Request, Server
    reqs = [Request((64, 64, 64), (3, 1, -2), dict(c=-0.7), 12, True, rid=0),
            Request((24, 24, 24), (0, 0, 0), dict(a=-0.3, c=-0.2), 6, True, rid=1),
            Request((37, 50, 29), (1, -3, 2), dict(n=0.2, seed=9, c=-0.3), 9, False, rid=2)]
    srv = Server(slots=1, max_size=(64, 64, 64), brick_capacity=4000, keep_outputs=True)
    try:
        for r in reqs:
            assert srv.submit(r)
        assert srv.drain(120)
        res = {r.rid: r for r in srv.results()}
        for r in reqs:
            _check_alone(srv, r, res[r.rid])
    finally:
        srv.close()


def test_admission_rejects_over_budget():
    from felt_b200.serving import Request, Server, reserve_bricks
    r = Request((64, 64, 64), (0, 0, 0), dict(c=-0.5), 10, False, "constant", rid=0)
    need = reserve_bricks(r, 2, (8, 8, 8))
    srv = Server(slots=4, max_size=(64, 64, 64), brick_capacity=int(1.5 * need))
    try:
        assert srv.submit(r)
        r2 = Request((64, 64, 64), (0, 0, 0), dict(c=-0.5), 10, False, "constant", rid=1)
        assert not srv.submit(r2)
        big = Request((128, 128, 128), (0, 0, 0), dict(c=-0.5), 2, False, rid=2)
        assert not srv.submit(big)  # larger than the slots' grids
        assert srv.drain(120)
        st = srv.stats()
        assert (st["admitted"], st["rejected"]) == (1, 2)
        # the reservation returned: the same request fits again
        assert srv.submit(r2)
        assert srv.drain(120)
    finally:
        srv.close()


def test_reservation_covers_real_brick_use():
    """The admission bound is an upper bound of the bricks a request really holds: one request
    at a time, the pool's peak use never exceeds its reservation."""
    from felt_b200.serving import Server
    for r in _requests(9, seed=11):
        srv = Server(slots=1, max_size=(64, 64, 64), brick_capacity=6000)
        try:
            need = srv.request_bricks(r)
            assert srv.submit(r)
            assert srv.drain(120)
            st = srv.stats()
            assert 0 < st["peak_used_bricks"] <= need, (r, st["peak_used_bricks"], need)
        finally:
            srv.close()
