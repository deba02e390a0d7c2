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
