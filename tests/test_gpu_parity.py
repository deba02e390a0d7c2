"""Parity of the device engine (libfelt_gpu.so via its C ABI) with the CPU oracle.

Layer lists, list order, partition lists, activation and backgrounds must be bit-exact (the
canonical dumps are compared word for word); FP32 distances must agree within 1e-5 absolute
(the stated tolerance) and in practice are bit-identical."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.dumps import first_difference
from tests.scenario import run_steps

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PHI_TOL = 1e-5


def _fb():
    import felt_b200
    return felt_b200


def _golden_global():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        cases = json.load(f)["surface"]
    return [c for c in cases if all(st[0] in ("seed", "update") for st in c["steps"])]


def assert_same(gpu, ora, where):
    d = first_difference(gpu.dump(), ora.dump())
    assert d is None, f"{where}: {d}"
    a, b = gpu.snapshot(), ora.snapshot()
    err = float(np.abs(a - b).max()) if a.size else 0.0
    assert err <= PHI_TOL, f"{where}: max |phi_gpu - phi_oracle| = {err}"


@pytest.mark.parametrize("case", _golden_global(), ids=lambda c: c["name"])
def test_golden_global_updates(case):
    fb = _fb()
    g = fb.Surface(case["size"], case["part"], case["layers"])
    o = O.Surface(case["size"], case["part"], case["layers"])
    for i, st in enumerate(case["steps"]):
        run_steps(g, [st])
        run_steps(o, [st])
        assert_same(g, o, f"step {i} {st}")
    if case["grid"]:
        np.testing.assert_allclose(g.snapshot().T.flatten(), np.array(case["grid"], np.float32),
                                   atol=1e-6)


def run_compare(size, part, L, seeds, schedule, every=1):
    fb = _fb()
    g = fb.Surface(size, part, L)
    o = O.Surface(size, part, L)
    for s in seeds:
        g.seed(s)
        o.seed(s)
    assert_same(g, o, "after seed")
    step = 0
    for n, kw in schedule:
        for _ in range(n):
            g.update(**kw)
            o.update(**kw)
            step += 1
            if step % every == 0:
                assert_same(g, o, f"step {step} {kw}")
    assert_same(g, o, f"final step {step}")
    return g, o


def test_c1_plain_64cubed():
    """Surface<3,2> 64^3 with 8^3 partitions, seed at the origin, 50 steps of speed -0.5."""
    run_compare((64, 64, 64), (8, 8, 8), 2, [(0, 0, 0)], [(50, dict(c=-0.5))], every=5)


def test_expand_then_contract_to_nothing_3d():
    run_compare((24, 24, 24), (4, 4, 4), 2, [(0, 0, 0)],
                [(6, dict(c=-1.0)), (10, dict(c=0.7))], every=1)


def test_curvature_and_noise_3d_L3():
    run_compare((48, 48, 48), (8, 8, 8), 3, [(0, 0, 0)],
                [(8, dict(c=-1.0)), (20, dict(a=-0.2, n=0.1, seed=7))], every=2)


def test_curvature_const_3d_uneven_partitions():
    run_compare((40, 24, 32), (16, 8, 16), 2, [(1, 0, -2)],
                [(6, dict(c=-0.8)), (12, dict(a=-0.3, c=0.1))], every=2)


def test_2d_multi_seed_merge():
    run_compare((96, 80), (16, 16), 2, [(-20, 0), (20, 5), (0, -25)],
                [(30, dict(c=-0.45)), (10, dict(a=-0.5, c=0.2))], every=3)


def test_2d_noise_L1():
    run_compare((64, 64), (8, 8), 1, [(3, -4)], [(25, dict(n=0.6, c=-0.3, seed=3))], every=1)


def test_consumed_grid_edges_3d():
    """The band reaches the grid edge and the whole grid is consumed (partitions deactivate
    with the inside background)."""
    run_compare((20, 20, 20), (5, 5, 5), 2, [(0, 0, 0)], [(25, dict(c=-1.0))], every=1)


def test_nonfinite_delta_reports_error():
    fb = _fb()
    g = fb.Surface((16, 16), (8, 8), 2)
    g.seed((0, 0))
    with pytest.raises(fb.FeltError) as ei:
        g.update(c=float("nan"))
    assert ei.value.code == -10


def test_determinism_two_runs():
    g1, _ = run_compare((32, 32, 32), (8, 8, 8), 2, [(0, 0, 0)], [(12, dict(a=-0.3, c=-0.4))],
                        every=12)
    g2, _ = run_compare((32, 32, 32), (8, 8, 8), 2, [(0, 0, 0)], [(12, dict(a=-0.3, c=-0.4))],
                        every=12)
    assert np.array_equal(g1.dump(), g2.dump())
    assert np.array_equal(g1.snapshot(), g2.snapshot())


def test_c2_shaped_16cubed_bricks_L3():
    """The headline workload's shape at a size the oracle finishes quickly: 16^3 partitions
    (4096-leaf bricks: split first pass, block-per-partition record passes, windowed flush),
    L=3, expansion then curvature + hashed noise."""
    run_compare((96, 96, 96), (16, 16, 16), 3, [(0, 0, 0)],
                [(20, dict(c=-1.0)), (16, dict(a=-0.2, n=0.1, seed=1234))], every=4)
