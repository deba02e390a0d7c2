"""The whole global update as one persistent launch (k_update_step) against the same update
launched one kernel per phase: every list, order, partition list and value must be the same, for
single surfaces, batches of uneven surfaces (including one the convergence cap stops), custom
functor halves and every launch-tuning knob. Its grid barriers wait a bounded time: a barrier
that cannot complete gives up with FG_ERR_TIMEOUT and leaves the surface usable."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.dumps import first_difference

pytestmark = pytest.mark.gpu


def _fb():
    import felt_b200
    return felt_b200


def _run(mode, size, part, L, seed, schedule, **tuning):
    fb = _fb()
    s = fb.Surface(size, part, L, launch_mode=mode, **tuning)
    s.seed(seed)
    states = []
    for n, kw in schedule:
        for _ in range(n):
            s.update(**kw)
        states.append((s.dump(), s.snapshot()))
    return s, states


CASES = [
    ((48, 48, 48), (8, 8, 8), 2, (0, 0, 0), [(6, dict(c=-1.0)), (10, dict(a=-0.3, c=-0.1))]),
    ((96, 96, 96), (16, 16, 16), 3, (2, -1, 0), [(12, dict(c=-1.0)), (6, dict(a=-0.2, n=0.1, seed=3))]),
    ((40, 24, 32), (16, 8, 16), 2, (1, 0, -2), [(6, dict(c=-0.8)), (8, dict(a=-0.3, c=0.1))]),
    ((120, 90), (16, 16), 2, (5, -3), [(20, dict(c=-0.6)), (10, dict(c=0.5))]),
    ((20, 20, 20), (5, 5, 5), 2, (0, 0, 0), [(25, dict(c=-1.0))]),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])))
def test_persistent_equals_per_phase(case):
    size, part, L, seed, sched = case
    a, sa = _run(1, size, part, L, seed, sched)
    b, sb = _run(2, size, part, L, seed, sched)
    assert a.tuning()["launch_mode"] == 1 and b.tuning()["launch_mode"] == 2
    for (da, pa), (db, pb) in zip(sa, sb):
        d = first_difference(da, db)
        assert d is None, d
        assert np.array_equal(pa, pb)
    assert a.node_updates() == b.node_updates()


def test_persistent_matches_oracle_with_polys():
    fb = _fb()
    size, part, L = (64, 64, 64), (8, 8, 8), 2
    g = fb.Surface(size, part, L, launch_mode=1)
    o = O.Surface(size, part, L)
    gp, op = fb.Polys(g), O.Polys(o)
    for s in (g, o):
        s.seed((0, 0, 0))
    for k in range(24):
        kw = dict(c=-0.7) if k < 12 else dict(a=-0.3, n=0.2, seed=k, c=0.05)
        for s, p in ((g, gp), (o, op)):
            s.update(**kw)
            p.notify()
        if k % 6 == 5:
            gp.march()
            op.march()
            assert gp.changes() == op.changes()
        d = first_difference(g.dump(), o.dump())
        assert d is None, f"step {k}: {d}"
    assert float(np.abs(g.snapshot() - o.snapshot()).max()) <= 1e-5


@pytest.mark.parametrize("tuning", [dict(dist_split=1), dict(dist_split=8),
                                    dict(record_passes=1), dict(record_passes=2),
                                    dict(blocks_per_sm=1), dict(blocks_per_sm=2)],
                         ids=lambda t: "-".join(f"{k}{v}" for k, v in t.items()))
def test_tuning_knobs_keep_results(tuning):
    size, part, L, seed, sched = CASES[1]
    ref, sref = _run(2, size, part, L, seed, sched)
    for mode in (1, 2):
        a, sa = _run(mode, size, part, L, seed, sched, **tuning)
        for (da, pa), (db, pb) in zip(sa, sref):
            assert first_difference(da, db) is None
            assert np.array_equal(pa, pb)


def test_batch_persistent_equals_per_phase_with_a_stopped_surface():
    """Batches of uneven surfaces, one of which the 64-iteration cap stops in both paths."""
    fb = _fb()
    sizes = [(48, 48, 48), (32, 32, 32), (40, 24, 48), (56, 56, 56)]
    centres = [(-19, 3, 18), (0, 0, 0), (2, -3, 1), (4, 4, -4)]
    speeds = [dict(a=-0.3, c=-0.5259483650318802), dict(a=-0.3, c=-0.2), dict(c=-0.6),
              dict(n=0.2, seed=7, c=-0.3)]
    out = []
    for mode in (1, 2):
        b = fb.Batch(sizes, (8, 8, 8), 2, launch_mode=mode)
        b.seed(centres)
        for _ in range(60):
            b.update(speeds)
            b.polys_notify()
        b.polys_march()
        out.append(([b.dump(i) for i in range(4)], [b.snapshot(i) for i in range(4)],
                    [b.stopped(i) for i in range(4)], b.polys_totals(), b.node_updates()))
    (da, pa, sa, ta, na), (db, pb, sb, tb, nb) = out
    assert sa == sb and sa[0] and not any(sa[1:])
    for i in range(4):
        assert first_difference(da[i], db[i]) is None, i
        assert np.array_equal(pa[i], pb[i])
    assert ta == tb and na == nb


def test_barrier_wait_gives_up_and_surface_stays_usable():
    """A barrier that can never complete (it waits for one block more than the launch has):
    every block gives up after the wait bound and the call reports FG_ERR_TIMEOUT; the kernel
    stopped before any work, so the surface then updates exactly as the oracle."""
    fb = _fb()
    size, part, L = (32, 32, 32), (8, 8, 8), 2
    g = fb.Surface(size, part, L, launch_mode=1)
    o = O.Surface(size, part, L)
    for s in (g, o):
        s.seed((0, 0, 0))
    for s in (g, o):
        s.update(c=-0.8)
    assert g.check_step_timeout(0.2) == -14
    for _ in range(5):
        for s in (g, o):
            s.update(a=-0.3, c=-0.3)
    assert first_difference(g.dump(), o.dump()) is None
    assert float(np.abs(g.snapshot() - o.snapshot()).max()) <= 1e-5
