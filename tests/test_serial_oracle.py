"""Surface::save / Surface::load (include/Felt/Surface.hpp:180-196) in the oracle: the
reference's own save/load test (test_Surface.cpp:464-500), round trips, and the file layout
(the isogrid through cereal's binary archive) checked against sizes computed independently."""
import json
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O
from tests.scenario import run_steps

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _serial_cases():
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        return json.load(f)["serial"]


def iso_state(s):
    """The isogrid as the file holds it: per partition its state and leaf lists, and the
    partition lists."""
    n, _, _ = s.partitions()
    nl = 2 * s.L + 1
    parts = [(s.partition_state(p), [s.layer_list(p, li) for li in range(nl)]) for p in range(n)]
    return parts, [s.partition_list(li) for li in range(nl)]


@pytest.mark.parametrize("case", _serial_cases(), ids=lambda c: c["name"])
def test_save_load_golden(case):
    s = O.Surface(case["size"], case["part"], case["layers"])
    run_steps(s, case["before"])
    t = O.Surface.load(s.save())
    assert np.array_equal(t.snapshot(), s.snapshot())
    run_steps(t, case["after"])
    np.testing.assert_allclose(t.snapshot().T.flatten(), np.array(case["grid"], np.float32),
                               atol=1e-6)


SCENES = [
    ((32, 32, 32), (5, 5, 5), 3, [(0, 0, 0)], [(4, dict(c=-1.0))]),
    ((40, 24), (8, 8), 2, [(0, 0)], [(6, dict(c=-1.0))]),
    ((17, 23, 19), (4, 4, 4), 1, [(1, -2, 0)], [(4, dict(c=-1.0))]),
    ((33, 29), (3, 5), 4, [(-3, 2), (6, -4)], [(5, dict(c=-0.8))]),
    ((24, 24, 24), (8, 8, 8), 2, [(0, 0, 0)], []),
]


def build(scene):
    size, part, L, seeds, schedule = scene
    s = O.Surface(size, part, L)
    for c in seeds:
        s.seed(c)
    for n, kw in schedule:
        for _ in range(n):
            s.update(**kw)
    return s


@pytest.mark.parametrize("si", range(len(SCENES)))
def test_oracle_round_trip(si):
    s = build(SCENES[si])
    data = s.save()
    t = O.Surface.load(data)
    assert (t.D, t.L, t.size, t.part) == (s.D, s.L, s.size, s.part)
    assert np.array_equal(t.snapshot(), s.snapshot())
    assert iso_state(t) == iso_state(s)
    assert t.save() == data
    for _ in range(3):
        s.update(a=-0.2, c=-0.3)
        t.update(a=-0.2, c=-0.3)
    assert np.array_equal(t.snapshot(), s.snapshot())
    assert t.save() == s.save()


def expected_empty_length(size, part, L):
    """File length of a surface with no active partition, from the layout: every child is an
    inactive Child (background, empty values, a leaf lookup with empty data and N empty lists,
    two size/offset triples)."""
    D, N = len(size), 2 * L + 1
    vec = 16 + 4 * D
    exact = all(s % p == 0 for s, p in zip(size, part))
    count = int(np.prod([s // p + (0 if exact else 1) for s, p in zip(size, part)]))
    child = 4 + 8 + 8 + 8 + (16 + 8 * N) + 6 * vec
    lookup = (16 + 8 * N) + 8 + count * (16 + 8 * N) + (16 + 8 * N) + 3 * vec
    return 4 + vec + child + 8 + count * child + lookup + 3 * vec + 3 * vec + 4 + 2 * vec


@pytest.mark.parametrize("size,part,L", [((16, 16), (4, 4), 2), ((9, 10, 11), (4, 4, 4), 3),
                                         ((20, 20, 20), (5, 5, 5), 1)])
def test_layout_of_an_empty_surface(size, part, L):
    s = O.Surface(size, part, L)
    data = s.save()
    assert len(data) == expected_empty_length(size, part, L)
    D = len(size)
    # background L+1, then the child size as an Eigen vector: rows, cols, length, values
    assert struct.unpack_from("<f", data, 0)[0] == float(L + 1)
    rows, cols, n = struct.unpack_from("<iiQ", data, 4)
    assert (rows, cols, n) == (D, 1, D)
    assert list(struct.unpack_from(f"<{D}i", data, 20)) == list(part)
    # the tail: grid size, offset, offset + size, dx = 1, pos_min, pos_max
    vec = 16 + 4 * D
    tail = data[len(data) - (5 * vec + 4):]
    size_v = struct.unpack_from(f"<{D}i", tail, 16)
    off_v = struct.unpack_from(f"<{D}i", tail, vec + 16)
    assert list(size_v) == list(size)
    assert list(off_v) == [int(-s / 2) for s in size]
    assert struct.unpack_from("<f", tail, 3 * vec)[0] == 1.0


def test_layout_of_a_seeded_surface():
    """A seed activates partitions: each adds its values (4 B per leaf), its leaf lookup (8 B
    per leaf) and its listed leaves (8 B each) to the empty file, and each partition-list entry
    adds 8 B."""
    size, part, L = (16, 16), (4, 4), 2
    s = O.Surface(size, part, L)
    s.seed((0, 0))
    s.update(c=-1.0)
    n, _, _ = s.partitions()
    bv = int(np.prod(part))
    nl = 2 * L + 1
    active = sum(s.partition_state(p)[0] for p in range(n))
    listed = sum(len(s.layer_list(p, li)) for p in range(n) for li in range(nl))
    plisted = sum(len(s.partition_list(li)) for li in range(nl))
    extra = active * bv * (4 + 8) + listed * 8 + plisted * 8
    assert len(s.save()) == expected_empty_length(size, part, L) + extra


def test_malformed_files_are_rejected():
    s = build(SCENES[1])
    data = bytearray(s.save())
    with pytest.raises(O.OracleError):
        O.Surface.load(bytes(data[:-3]))
    with pytest.raises(O.OracleError):
        O.Surface.load(bytes(data) + b"\0")
    # the first leaf list entry of the first active partition, pointed at another leaf
    bad = bytearray(data)
    found = False
    D, N = 2, 5
    vec = 16 + 4 * D
    child_empty = 4 + 8 + 8 + 8 + (16 + 8 * N) + 6 * vec
    at = 4 + vec + child_empty + 8
    nparts = s.partitions()[0]
    bv = 64
    for p in range(nparts):
        active, _ = s.partition_state(p)
        if not active:
            at += child_empty
            continue
        lists = [s.layer_list(p, li) for li in range(N)]
        pos = at + 4 + 8 + 4 * bv + 8 + 8 + 8 * bv + 16
        for li in range(N):
            if lists[li]:
                entry = pos + 8
                (v,) = struct.unpack_from("<Q", bad, entry)
                struct.pack_into("<Q", bad, entry, (v + 1) % bv)
                found = True
                break
            pos += 8
        break
    assert found
    with pytest.raises(O.OracleError):
        O.Surface.load(bytes(bad))
