"""Parity of the device Polys (marching squares/cubes) with the oracle: pending/done partition
lists, vertex counts, vertex order and simplex index triplets bit-exact; vertex positions and
normals within 1e-5 absolute (the stated tolerance)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.scenario import child_index, run_steps

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VTX_TOL = 1e-5


def _fb():
    import felt_b200
    return felt_b200


def compare_polys(gp, op, nparts, where):
    assert gp.changes() == op.changes(), f"{where}: changes differ"
    tv = ts = 0
    for p in range(nparts):
        ov, os_, _ = op.partition(p)
        tv += ov.shape[0]
        ts += os_.shape[0]
    assert gp.totals() == (tv, ts), f"{where}: totals {gp.totals()} vs {(tv, ts)}"
    for p in range(nparts):
        gv, gs, ga = gp.partition(p)
        ov, os_, oa = op.partition(p)
        assert ga == oa, f"{where}: partition {p} active {ga} vs {oa}"
        assert gv.shape == ov.shape, f"{where}: partition {p} vertices {gv.shape} vs {ov.shape}"
        assert gs.shape == os_.shape, f"{where}: partition {p} simplices {gs.shape} vs {os_.shape}"
        assert np.array_equal(gs, os_), f"{where}: partition {p} simplex indices differ"
        if gv.size:
            err = float(np.abs(gv - ov).max())
            assert err <= VTX_TOL, f"{where}: partition {p} vertex error {err}"


def run_polys(size, part, L, seeds, schedule, march_every=1, invalidate_at=(), vertex_capacity=0):
    fb = _fb()
    g = fb.Surface(size, part, L, vertex_capacity=vertex_capacity)
    o = O.Surface(size, part, L)
    gp = fb.Polys(g)
    op = O.Polys(o)
    for s in seeds:
        g.seed(s)
        o.seed(s)
    nparts = o.partitions()[0]
    step = 0
    for n, kw in schedule:
        for _ in range(n):
            g.update(**kw)
            o.update(**kw)
            gp.notify()
            op.notify()
            step += 1
            if step in invalidate_at:
                gp.invalidate()
                op.invalidate()
            if step % march_every == 0:
                gp.march()
                op.march()
                compare_polys(gp, op, nparts, f"step {step}")
    return g, gp


def test_polys_3d_expand_contract():
    run_polys((32, 32, 32), (8, 8, 8), 2, [(0, 0, 0)],
              [(10, dict(c=-0.7)), (6, dict(c=0.6))], march_every=1)


def test_polys_3d_curvature_noise_L3():
    run_polys((40, 40, 40), (8, 8, 8), 3, [(0, 0, 0)],
              [(6, dict(c=-1.0)), (10, dict(a=-0.2, n=0.1, seed=11))], march_every=2,
              invalidate_at=(9,))


def test_polys_2d_saddles_and_merge():
    run_polys((64, 48), (8, 8), 2, [(-10, 0), (10, 3)],
              [(12, dict(c=-0.55)), (8, dict(a=-0.4, c=0.15))], march_every=1)


def test_polys_3d_16cubed_bricks_noise():
    """16^3 bricks: the staged box of the march is 17^3 and most cells' corners lie inside it."""
    run_polys((80, 80, 80), (16, 16, 16), 3, [(0, 0, 0)],
              [(16, dict(c=-1.0)), (8, dict(a=-0.2, n=0.1, seed=99))], march_every=4)


def test_polys_arena_growth_and_compaction():
    """A 64-vertex initial arena: marches overflow and are retried after growth, and the arena
    is compacted (device-side offsets, alternating arenas) many times; the geometry stays the
    oracle's."""
    run_polys((40, 40, 40), (8, 8, 8), 2, [(0, 0, 0)],
              [(10, dict(c=-1.0)), (10, dict(a=-0.3, n=0.2, seed=5, c=-0.1))], march_every=1,
              vertex_capacity=64)


def test_polys_3d_uneven_partitions():
    run_polys((30, 18, 26), (16, 8, 16), 2, [(0, 0, 0)],
              [(7, dict(c=-0.8)), (4, dict(a=-0.3, c=-0.1))], march_every=1)


def _golden_poly():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        return json.load(f)["poly"]


@pytest.mark.parametrize("case", _golden_poly(), ids=lambda c: c["name"])
def test_golden_poly_on_gpu(case):
    fb = _fb()
    s = fb.Surface(case["size"], case["part"], case["layers"])
    p = fb.Polys(s)
    run_steps(s, case["steps"])
    _, ccount, coff = s.partitions()
    pc = child_index(case["partition"], ccount, coff)
    if case["name"].startswith("poly_single"):
        p.march_partition(pc)
    else:
        p.notify()
        p.march()
    vtx, spx, active = p.partition(pc)
    assert active
    D = len(case["size"])
    assert len(vtx) == case["nvtx"] and len(spx) == case["nspx"]
    for row in case.get("pos") or []:
        np.testing.assert_allclose(vtx[row[0], :D], row[1:], atol=1e-5)
    for row in case.get("norm") or []:
        np.testing.assert_allclose(vtx[row[0], D:2 * D], row[1:], atol=1e-5)
    for row in case.get("spx") or []:
        assert list(spx[row[0]]) == row[1:]
