"""Serving: a request's result is the same alone as in a mix. Requests of one wave share kernel
launches and finish at different steps; each finished one is paused, and its state (lists,
orders, values, polygons) equals the oracle's run of that request alone."""
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


def test_server_results_equal_alone():
    from felt_b200.serving import Request, Server
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(12):
        e = int(rng.choice([32, 40, 48]))
        kind = ["constant", "curvature", "noise"][k % 3]
        sp = {"constant": dict(c=-0.4), "curvature": dict(a=-0.3, c=-0.2),
              "noise": dict(n=0.2, seed=11, c=-0.2)}[kind]
        c = tuple(int(x) for x in rng.integers(-4, 5, size=3))
        reqs.append(Request((e, e, e), c, sp, int(rng.integers(1, 12)), bool(k % 2), kind,
                            rid=k))
    srv = Server(workers=2, tick=0.001, max_wave=5, keep_outputs=True)
    try:
        for r in reqs:
            r.arrival = srv.now()
            assert srv.submit(r)
        assert srv.drain(300)
        res = {r.rid: r for r in srv.results()}
    finally:
        srv.close()
    assert sorted(res) == list(range(len(reqs)))
    for r in reqs:
        o, _ = _oracle_alone(r.size, r.centre, r.speed, r.steps)
        d = first_difference(res[r.rid].dump, o.dump())
        assert d is None, f"request {r.rid}: {d}"
        assert res[r.rid].latency >= 0


def test_admission_rejects_over_budget():
    from felt_b200.serving import Request, Server, reserve_bytes
    r = Request((64, 64, 64), (0, 0, 0), dict(c=-0.5), 10, False, "constant", rid=0)
    need = reserve_bytes(r, 2, (8, 8, 8))[1]
    srv = Server(budget_bytes=1.5 * need, workers=1, tick=0.001)
    try:
        assert srv.submit(r)
        r2 = Request((64, 64, 64), (0, 0, 0), dict(c=-0.5), 10, False, "constant", rid=1)
        assert not srv.submit(r2)
        assert srv.drain(120)
        assert (srv.admitted, srv.rejected) == (1, 1)
    finally:
        srv.close()
