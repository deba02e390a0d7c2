"""The whole global update as one CUDA graph (launch mode 1, the default) against the same update
with every kernel launched one by one from the host (launch mode 2, no graphs): every list, order, partition
list and value must be the same, for single surfaces, batches of uneven surfaces (including one
the convergence cap stops), alternating speed kinds (which select different captured graphs) and
every launch-tuning knob; both count the same kernels per step."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.dumps import first_difference
from tests.test_gpu_local import _zero_layer_positions

pytestmark = pytest.mark.gpu


def _fb():
    import felt_b200
    return felt_b200


def _run(mode, size, part, L, seed, schedule, **tuning):
    fb = _fb()
    s = fb.Surface(size, part, L, launch_mode=mode, **tuning)
    s.seed(seed)
    states, launches = [], []
    for n, kw in schedule:
        for _ in range(n):
            l0 = fb.launch_count()
            s.update(**kw)
            launches.append((fb.launch_count() - l0, s.iterations()))
        states.append((s.dump(), s.snapshot()))
    return s, states, launches


CASES = [
    ((48, 48, 48), (8, 8, 8), 2, (0, 0, 0), [(6, dict(c=-1.0)), (10, dict(a=-0.3, c=-0.1))]),
    ((96, 96, 96), (16, 16, 16), 3, (2, -1, 0), [(12, dict(c=-1.0)), (6, dict(a=-0.2, n=0.1, seed=3))]),
    ((40, 24, 32), (16, 8, 16), 2, (1, 0, -2), [(6, dict(c=-0.8)), (8, dict(a=-0.3, c=0.1))]),
    ((120, 90), (16, 16), 2, (5, -3), [(20, dict(c=-0.6)), (10, dict(c=0.5))]),
    ((20, 20, 20), (5, 5, 5), 2, (0, 0, 0), [(25, dict(c=-1.0))]),
    ((32, 32, 32), (8, 8, 8), 2, (0, 0, 0),
     [(4, dict(c=-1.0)), (1, dict(a=-0.3, c=-0.2)), (1, dict(c=-0.4)),
      (2, dict(a=-0.2, c=-0.1)), (3, dict(n=0.2, seed=1, c=-0.3)), (1, dict(a=-0.3, c=0.1)),
      (2, dict(c=-0.5))]),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])))
def test_step_graph_equals_phase_by_phase(case):
    size, part, L, seed, sched = case
    a, sa, la = _run(1, size, part, L, seed, sched)
    b, sb, lb = _run(2, size, part, L, seed, sched)
    assert a.tuning()["launch_mode"] == 1 and b.tuning()["launch_mode"] == 2
    for (da, pa), (db, pb) in zip(sa, sb):
        d = first_difference(da, db)
        assert d is None, d
        assert np.array_equal(pa, pb)
    assert a.node_updates() == b.node_updates()
    # the same kernels run either way (the graph's are counted when it replays), plus the
    # device loop's control kernels: one to start it and one test per further iteration
    assert [it for _, it in la] == [it for _, it in lb]
    assert [na - nb for (na, _), (nb, _) in zip(la, lb)] == [it for _, it in la]


def test_step_graph_matches_oracle_with_polys():
    fb = _fb()
    size, part, L = (64, 64, 64), (8, 8, 8), 2
    g = fb.Surface(size, part, L)
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


def test_step_graph_between_local_updates():
    """Global updates (graph) interleaved with local updates (host-launched) and bounded
    updates: the host's record of which grids need resets stays right across both."""
    fb = _fb()
    size, part, L = (40, 40, 40), (8, 8, 8), 2
    g = fb.Surface(size, part, L)
    o = O.Surface(size, part, L)
    for s in (g, o):
        s.seed((0, 0, 0))
    for k in range(8):
        for s in (g, o):
            s.update(c=-0.6)
        if k % 3 == 1:
            zs = _zero_layer_positions(o)
            picks = [zs[(i * 7919) % len(zs)] for i in range(5)]
            for s in (g, o):
                s.update_start()
                for i, p in enumerate(picks):
                    s.delta(p, -0.3 + 0.1 * i)
                s.update_end()
        if k % 3 == 2:
            for s in (g, o):
                s.update_bounded((-3, -3, -3), (3, 3, 3), a=-0.2, c=-0.1)
        d = first_difference(g.dump(), o.dump())
        assert d is None, f"step {k}: {d}"
    assert float(np.abs(g.snapshot() - o.snapshot()).max()) <= 1e-5


@pytest.mark.parametrize("tuning", [dict(dist_split=1), dict(dist_split=8),
                                    dict(record_passes=1), dict(record_passes=2),
                                    dict(delta_kernel=1), dict(delta_kernel=2),
                                    dict(fuse_passes=1), dict(fuse_passes=2),
                                    dict(fuse_passes=3)],
                         ids=lambda t: "-".join(f"{k}{v}" for k, v in t.items()))
def test_tuning_knobs_keep_results(tuning):
    size, part, L, seed, sched = CASES[1]
    ref, sref, _ = _run(2, size, part, L, seed, sched)
    for mode in (1, 2):
        a, sa, _ = _run(mode, size, part, L, seed, sched, **tuning)
        for k, v in tuning.items():
            assert a.tuning()[k] == v
        for (da, pa), (db, pb) in zip(sa, sref):
            assert first_difference(da, db) is None
            assert np.array_equal(pa, pb)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])))
@pytest.mark.parametrize("mode", [1, 2])
def test_tiled_passes_match_oracle(case, mode):
    """fuse_passes 3 (every distance pass of a brick in shared memory, the brick staged with a
    halo of 2L nodes) against the oracle: lists, orders and values after every segment."""
    size, part, L, seed, sched = case
    g, sg, _ = _run(mode, size, part, L, seed, sched, fuse_passes=3)
    assert g.tuning()["fuse_passes"] == 3
    o = O.Surface(size, part, L)
    o.seed(seed)
    for (n, kw), (dg, pg) in zip(sched, sg):
        for _ in range(n):
            o.update(**kw)
        d = first_difference(dg, o.dump())
        assert d is None, d
        assert float(np.abs(pg - o.snapshot()).max()) <= 1e-5


def test_batch_step_graph_equals_phase_by_phase_with_a_stopped_surface():
    """Batches of uneven surfaces, one of which the 64-iteration cap stops in both modes."""
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


def test_autotune_picks_a_candidate_and_caches_it(tmp_path, monkeypatch):
    fb = _fb()
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("FELT_TUNE_CACHE", str(cache))
    part, L = (16, 16, 16), 3
    cand = fb.autotune_candidates(part)
    assert (1, 1) in cand and len(cand) == len(set(cand))
    t = fb.autotune(part, L, force=True)
    assert (t["dist_split"], t["record_passes"]) in cand
    assert sorted(t["ms"]) == sorted(cand) and all(v > 0 for v in t["ms"].values())
    assert t["ms"][(t["dist_split"], t["record_passes"])] == min(t["ms"].values())
    # cached: no timing the second time, the same choice, and the file holds it
    again = fb.autotune(part, L)
    assert again["ms"] == {} and again["dist_split"] == t["dist_split"]
    line = cache.read_text().split()
    assert line[1:3] == [str(t["dist_split"]), str(t["record_passes"])]
    # a surface created with autotune runs the tuned shapes and the same update as any other
    size, _, _, seed, sched = CASES[1]
    a, sa, _ = _run(1, size, part, L, seed, sched, autotune=True)
    assert a.tuning()["dist_split"] == t["dist_split"]
    assert a.tuning()["record_passes"] == t["record_passes"]
    b, sb, _ = _run(2, size, part, L, seed, sched, dist_split=1, record_passes=1)
    for (da, pa), (db, pb) in zip(sa, sb):
        assert first_difference(da, db) is None
        assert np.array_equal(pa, pb)


@pytest.mark.parametrize("case", [((33, 33, 33), (6, 6, 6)), ((37, 29, 41), (5, 5, 5)),
                                  ((44, 36, 52), (8, 8, 8)), ((50, 34), (16, 16))],
                         ids=lambda c: "x".join(map(str, c[0])) + "_p" + str(c[1][0]))
def test_staged_curvature_on_partial_and_odd_bricks(case):
    """The staged curvature speed copies whole brick rows in bulk where they are a multiple of
    16 bytes and lie inside the grid, and loads the rest node by node (rows of 5 or 6 floats,
    rows that leave a partial grid): both routes against the oracle."""
    fb = _fb()
    size, part = case
    D = len(size)
    g = fb.Surface(size, part, 2, delta_kernel=2)
    o = O.Surface(size, part, 2)
    seed = (1, -2, 0)[:D]
    for s in (g, o):
        s.seed(seed)
    for k in range(10):
        kw = dict(c=-0.8) if k < 4 else dict(a=-0.3, n=0.1, seed=k, c=-0.2)
        for s in (g, o):
            s.update(**kw)
        d = first_difference(g.dump(), o.dump())
        assert d is None, f"step {k}: {d}"
    assert float(np.abs(g.snapshot() - o.snapshot()).max()) <= 1e-5
