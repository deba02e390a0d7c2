"""Parity of the device local update (update_start / delta / update_end, calc_affected) and the
bounded update with the oracle: every golden scenario of the reference (global, local and
bounded steps) replayed on both, plus randomised local edits. Lists, list order, affected
lookups and activation bit-exact; distances within 1e-5 (in practice identical)."""
import os
import random

import numpy as np
import pytest

from oracle import oracle as O
from tests.dumps import first_difference
from tests.scenario import affected_positions, run_steps

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _fb():
    import felt_b200
    return felt_b200


def _golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        return json.load(f)["surface"]


def assert_same(g, o, where):
    d = first_difference(g.dump(), o.dump())
    assert d is None, f"{where}: {d}"
    err = float(np.abs(g.snapshot() - o.snapshot()).max())
    assert err <= 1e-5, f"{where}: max |phi_gpu - phi_oracle| = {err}"
    L = o.L
    for li in range(2 * L + 1):
        assert g.affected_partitions(li) == o.affected_partitions(li), f"{where}: affected {li}"
        for p in o.affected_partitions(li):
            assert g.affected_list(p, li) == o.affected_list(p, li), f"{where}: affected {p},{li}"


def _group(steps):
    """Groups update_start..update_end into one unit so comparisons happen between updates."""
    out, cur = [], None
    for st in steps:
        if st[0] == "update_start":
            cur = [st]
        elif cur is not None:
            cur.append(st)
            if st[0] == "update_end":
                out.append(cur)
                cur = None
        else:
            out.append([st])
    return out


@pytest.mark.parametrize("case", _golden(), ids=lambda c: c["name"])
def test_golden_scenarios_on_gpu(case):
    fb = _fb()
    g = fb.Surface(case["size"], case["part"], case["layers"])
    o = O.Surface(case["size"], case["part"], case["layers"])
    for i, unit in enumerate(_group(case["steps"])):
        run_steps(g, unit)
        run_steps(o, unit)
        assert_same(g, o, f"unit {i} {unit[0][0]}")
    if case.get("grid"):
        np.testing.assert_allclose(g.snapshot().T.flatten(),
                                   np.array(case["grid"], np.float32), atol=1e-6)
    for lid, want in (case.get("affected") or {}).items():
        assert sorted(affected_positions(g, int(lid) + case["layers"])) == sorted(want)


def _zero_layer_positions(o):
    """World positions of the oracle's zero-layer leaves."""
    L, D = o.L, o.D
    _, ccount, _ = o.partitions()
    out = []
    for p in o.partition_list(L):
        c, r = [0] * D, p
        for a in range(D - 1, -1, -1):
            c[a] = r % ccount[a]
            r //= ccount[a]
        org = [c[a] * o.part[a] + int(-o.size[a] / 2) for a in range(D)]
        for leaf in o.layer_list(p, L):
            q, r = [0] * D, leaf
            for a in range(D - 1, -1, -1):
                q[a] = r % o.part[a]
                r //= o.part[a]
            out.append([org[a] + q[a] for a in range(D)])
    return out


@pytest.mark.parametrize("dims,L", [(2, 2), (3, 2), (3, 3), (2, 1)])
def test_random_local_edits(dims, L):
    fb = _fb()
    rng = random.Random(1000 + 10 * dims + L)
    size = (40, 36) if dims == 2 else (24, 20, 22)
    part = (8, 8) if dims == 2 else (4, 4, 4)
    g = fb.Surface(size, part, L)
    o = O.Surface(size, part, L)
    for s in (g, o):
        s.seed((0,) * dims)
        for _ in range(4):
            s.update(c=-0.9)
    assert_same(g, o, "setup")
    for it in range(12):
        zs = _zero_layer_positions(o)
        k = rng.randint(1, min(6, len(zs)))
        picks = rng.sample(zs, k)
        if rng.random() < 0.3:
            picks.append(picks[0])  # repeated delta at one leaf: the last value wins
        vals = [rng.uniform(-0.95, 0.95) for _ in picks]
        for s in (g, o):
            s.update_start()
            for p, v in zip(picks, vals):
                s.delta(p, v)
            s.update_end()
        assert_same(g, o, f"edit {it}")


def test_bounded_updates_with_curvature():
    fb = _fb()
    g = fb.Surface((32, 32, 32), (8, 8, 8), 2)
    o = O.Surface((32, 32, 32), (8, 8, 8), 2)
    for s in (g, o):
        s.seed((0, 0, 0))
        for _ in range(5):
            s.update(c=-1.0)
    boxes = [((-6, -6, -6), (6, 0, 6)), ((0, 0, 0), (100, 100, 100)), ((-100, -3, -2), (2, 3, 4))]
    for i, (lo, hi) in enumerate(boxes):
        for s in (g, o):
            s.update_bounded(lo, hi, a=-0.3, c=-0.2)
        assert_same(g, o, f"box {i}")
