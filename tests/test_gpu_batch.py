"""A batch of independent surfaces advanced by shared kernel launches gives, per surface,
exactly what a separate surface (checked against the oracle) gives: lists, orders, values,
polygonisation."""
import random

import numpy as np
import pytest

from oracle import oracle as O
from tests.dumps import first_difference

pytestmark = pytest.mark.gpu


def _run_batch(D, L, part, sizes, centres, speeds_per_step, march_every=1):
    import felt_b200 as fb
    b = fb.Batch(sizes, part, L)
    b.seed(centres)
    os_ = [O.Surface(sz, part, L) for sz in sizes]
    ops = [O.Polys(o) for o in os_]
    for o, c in zip(os_, centres):
        o.seed(c)
    for step, speeds in enumerate(speeds_per_step):
        b.update(speeds)
        b.polys_notify()
        for o, op, sp in zip(os_, ops, speeds):
            o.update(**sp)
            op.notify()
        march = march_every and (step + 1) % march_every == 0
        if march:
            b.polys_march()
            for op in ops:
                op.march()
        for i, o in enumerate(os_):
            d = first_difference(b.dump(i), o.dump())
            assert d is None, f"step {step} surface {i}: {d}"
            err = float(np.abs(b.snapshot(i) - o.snapshot()).max())
            assert err <= 1e-5, f"step {step} surface {i}: phi error {err}"
            if march:
                assert b.polys_changes(i) == ops[i].changes(), f"step {step} surface {i} changes"
                for p in ops[i].changes():
                    gv, gs, ga = b.polys_partition(i, p)
                    ov, os2, oa = ops[i].partition(p)
                    assert ga == oa and np.array_equal(gs, os2), f"surface {i} partition {p}"
                    if ov.size:
                        assert float(np.abs(gv - ov).max()) <= 1e-5
        if march:
            tv = ts = 0
            for o, op in zip(os_, ops):
                for p in range(o.partitions()[0]):
                    ov, os2, _ = op.partition(p)
                    tv += ov.shape[0]
                    ts += os2.shape[0]
            assert b.polys_totals() == (tv, ts), f"step {step} totals"
    return b


def test_batch_2d_uneven_sizes_and_speeds():
    rng = random.Random(7)
    sizes = [(48, 48), (64, 40), (33, 57), (80, 80), (40, 64)]
    centres = [(rng.randint(-8, 8), rng.randint(-8, 8)) for _ in sizes]
    cs = [rng.uniform(-0.8, -0.2) for _ in sizes]
    steps = [[dict(c=c) for c in cs] for _ in range(20)]
    _run_batch(2, 2, (16, 16), sizes, centres, steps, march_every=1)


def test_oscillating_surface_stops_at_the_same_step():
    """Anti-diffusive curvature speed drives this surface into the grid edge, where the
    reference's unbounded convergence loop would cycle forever; the device engine and the
    oracle both stop it after the same number of iterations in the same update, and in a
    batch only that surface stops."""
    import felt_b200 as fb
    size, centre, c = (48, 48, 48), (-19, 3, 18), -0.5259483650318802
    g = fb.Surface(size, (8, 8, 8), 2)
    o = O.Surface(size, (8, 8, 8), 2)
    g.seed(centre)
    o.seed(centre)
    failed_at = None
    for step in range(70):
        try:
            o.update(a=-0.3, c=c)
        except O.OracleError as e:
            assert e.code == -14
            failed_at = step
            with pytest.raises(fb.FeltError) as ei:
                g.update(a=-0.3, c=c)
            assert ei.value.code == -14
            break
        g.update(a=-0.3, c=c)
        assert first_difference(g.dump(), o.dump()) is None, f"step {step}"
    assert failed_at is not None
    with pytest.raises(fb.FeltError) as ei:
        g.update(a=-0.3, c=c)
    assert ei.value.code == -15
    # in a batch the other surface carries on, identical to its own oracle run
    b = fb.Batch([size, (32, 32, 32)], (8, 8, 8), 2)
    b.seed([centre, (0, 0, 0)])
    o2 = O.Surface((32, 32, 32), (8, 8, 8), 2)
    o2.seed((0, 0, 0))
    for step in range(failed_at + 3):
        b.update([dict(a=-0.3, c=c), dict(a=-0.3, c=-0.2)])
        o2.update(a=-0.3, c=-0.2)
        assert b.stopped(0) == (step >= failed_at)
        assert not b.stopped(1)
        assert first_difference(b.dump(1), o2.dump()) is None, f"batch step {step}"


def test_batch_3d_curvature_mixed_contraction():
    rng = random.Random(11)
    sizes = [(32, 32, 32), (48, 48, 48), (24, 32, 40), (32, 32, 32)]
    centres = [(0, 0, 0), (2, -3, 1), (0, 1, 0), (-1, 0, 2)]
    cs = [-0.6, -0.2, 0.3, -0.45]
    steps = [[dict(c=-1.0)] * len(sizes)] * 3
    steps += [[dict(a=-0.3, c=c) for c in cs] for _ in range(10)]
    _run_batch(3, 2, (8, 8, 8), sizes, centres, steps, march_every=3)
