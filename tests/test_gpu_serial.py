"""Surface::save / Surface::load (include/Felt/Surface.hpp:180-196) on the device: the file a
device surface writes is byte for byte the oracle's for the same surface; a file from either
side loads into the other with the same isogrid, and both go on updating identically."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.scenario import run_steps
from tests.test_serial_oracle import SCENES, iso_state

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _fb():
    import felt_b200
    return felt_b200


def build_both(scene):
    fb = _fb()
    size, part, L, seeds, schedule = scene
    g = fb.Surface(size, part, L)
    o = O.Surface(size, part, L)
    for c in seeds:
        g.seed(c)
        o.seed(c)
    for n, kw in schedule:
        for _ in range(n):
            g.update(**kw)
            o.update(**kw)
    return g, o


@pytest.mark.parametrize("si", range(len(SCENES)))
def test_device_file_equals_oracle_file(si):
    g, o = build_both(SCENES[si])
    assert g.save() == o.save()


@pytest.mark.parametrize("si", range(len(SCENES)))
def test_load_either_way_then_update(si):
    fb = _fb()
    g, o = build_both(SCENES[si])
    data = o.save()
    g2 = fb.Surface.load(data)
    assert (g2.D, g2.L, g2.size, g2.part) == (o.D, o.L, o.size, o.part)
    assert np.array_equal(g2.snapshot(), o.snapshot())
    assert iso_state(g2) == iso_state(o)
    assert g2.save() == data
    o2 = O.Surface.load(g.save())
    for _ in range(4):
        for s in (g2, o2, o):
            s.update(a=-0.2, c=-0.3)
    assert np.array_equal(g2.snapshot(), o.snapshot())
    assert g2.save() == o.save() == o2.save()


def test_save_load_golden_device():
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        case = json.load(f)["serial"][0]
    fb = _fb()
    g = fb.Surface(case["size"], case["part"], case["layers"])
    run_steps(g, case["before"])
    t = fb.Surface.load(g.save())
    assert np.array_equal(t.snapshot(), g.snapshot())
    run_steps(t, case["after"])
    np.testing.assert_allclose(t.snapshot().T.flatten(), np.array(case["grid"], np.float32),
                               atol=1e-6)


def test_loaded_surface_polygonises_like_the_original():
    fb = _fb()
    g, o = build_both(SCENES[0])
    t = fb.Surface.load(g.save())
    p, q = fb.Polys(g), fb.Polys(t)
    p.invalidate()
    q.invalidate()
    p.march()
    q.march()
    assert p.totals() == q.totals()
    n, _, _ = g.partitions()
    for part in range(n):
        a, b = p.partition(part), q.partition(part)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_malformed_and_oversized_files_are_rejected():
    fb = _fb()
    g, o = build_both(SCENES[1])
    data = g.save()
    for bad in (data[:-5], data + b"\0", data[:40]):
        with pytest.raises(fb.FeltError) as ei:
            fb.Surface.load(bad)
        assert ei.value.code == -1
    # a value moved out of its listed layer
    t = fb.Surface.load(data)
    raw = bytearray(data)
    D, N = 2, 5
    vec = 16 + 4 * D
    child_empty = 4 + 8 + 8 + 8 + (16 + 8 * N) + 6 * vec
    at = 4 + vec + child_empty + 8
    n, _, _ = g.partitions()
    for part in range(n):
        if g.partition_state(part)[0]:
            lists = [g.layer_list(part, li) for li in range(N)]
            leaf = lists[N // 2][0]  # a zero-layer leaf
            off = at + 4 + 8 + 4 * leaf
            raw[off:off + 4] = np.float32(2.0).tobytes()
            break
        at += child_empty
    with pytest.raises(fb.FeltError) as ei:
        fb.Surface.load(bytes(raw))
    assert ei.value.code == -1
    # a pool too small for the file's active partitions
    with pytest.raises(fb.FeltError) as ei:
        fb.Surface.load(data, brick_capacity=1)
    assert ei.value.code == -4
    assert np.array_equal(t.snapshot(), g.snapshot())


BATCH_SIZES = [(32, 32, 32), (40, 24, 32), (24, 24, 24)]
BATCH_CENTRES = [(0, 0, 0), (3, -2, 1), (-1, 1, 0)]
BATCH_SPEEDS = [dict(c=-1.0), dict(c=-0.7, n=0.3, seed=4), dict(a=-0.3, c=-0.5)]


def _batch_and_oracles(steps):
    fb = _fb()
    part, L = (8, 8, 8), 2
    b = fb.Batch(BATCH_SIZES, part, L)
    b.seed(BATCH_CENTRES)
    os_ = [O.Surface(sz, part, L) for sz in BATCH_SIZES]
    for o, c in zip(os_, BATCH_CENTRES):
        o.seed(c)
    for _ in range(steps):
        b.update(BATCH_SPEEDS)
        for o, sp in zip(os_, BATCH_SPEEDS):
            o.update(**sp)
    return b, os_


def test_batch_save_equals_oracle_file():
    b, os_ = _batch_and_oracles(5)
    for i, o in enumerate(os_):
        assert b.save(i) == o.save(), f"surface {i}"


def test_batch_restore_then_update():
    """Checkpoint every surface of a batch, restore the files into a batch that was never
    seeded (in another order, so each surface lands in bricks that another surface's data
    held in the first batch), and advance both batches: every surface stays equal to its
    oracle."""
    fb = _fb()
    b, os_ = _batch_and_oracles(4)
    files = [b.save(i) for i in range(3)]
    c = fb.Batch(BATCH_SIZES, (8, 8, 8), 2)
    for i in (2, 0, 1):
        c.restore(i, files[i])
    for i, o in enumerate(os_):
        assert np.array_equal(c.snapshot(i), o.snapshot())
        assert c.save(i) == files[i]
    for _ in range(4):
        b.update(BATCH_SPEEDS)
        c.update(BATCH_SPEEDS)
        for o, sp in zip(os_, BATCH_SPEEDS):
            o.update(**sp)
    for i, o in enumerate(os_):
        assert np.array_equal(c.snapshot(i), o.snapshot()), f"surface {i}"
        assert c.save(i) == b.save(i) == o.save(), f"surface {i}"


def test_batch_restore_from_a_single_surface_file():
    """A file written by a single surface (or the oracle) restores into a batch position of
    the same grid, next to surfaces that keep running."""
    fb = _fb()
    part, L = (8, 8, 8), 2
    o = O.Surface((24, 24, 24), part, L)
    o.seed((2, 2, -3))
    for _ in range(5):
        o.update(c=-1.0)
    b = fb.Batch([(32, 32, 32), (24, 24, 24)], part, L)
    b.seed([(0, 0, 0), (0, 0, 0)])
    with pytest.raises(fb.FeltError):  # surface 1 is seeded: not empty
        b.restore(1, o.save())
    with pytest.raises(fb.FeltError):  # surface 0 has another grid size
        b.restore(0, o.save())
    e = fb.Batch([(32, 32, 32), (24, 24, 24)], part, L)
    e.restore(1, fb.Surface.load(o.save()).save())
    with pytest.raises(fb.FeltError):  # restored: no longer empty
        e.restore(1, o.save())
    for _ in range(3):
        e.update([dict(c=-1.0), dict(c=-1.0)])
        o.update(c=-1.0)
    assert np.array_equal(e.snapshot(1), o.snapshot())
    assert not np.any(e.snapshot(0) < 3)  # the never-seeded surface stays background
    with pytest.raises(fb.FeltError):  # a truncated file
        e.restore(0, b.save(0)[:-5])
    e.restore(0, b.save(0))
    assert np.array_equal(e.snapshot(0), b.snapshot(0))
