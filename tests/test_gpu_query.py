"""The isogrid's Numeric API from the host (fg_query, fg_query_nodes: get, curv, divergence,
inside and the five gradients of NumericMixin.hpp:72-481) against the oracle, bit for bit, at
nodes and at real positions, on single surfaces and a batch."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SCALARS = ["get", "curv", "divergence"]
VECTORS = ["grad", "gradF", "gradB", "gradC", "gradE"]


def _fb():
    import felt_b200
    return felt_b200


def _both(size, part, L, steps):
    fb = _fb()
    g, o = fb.Surface(size, part, L), O.Surface(size, part, L)
    for s in (g, o):
        s.seed(tuple(0 for _ in size))
        for _ in range(steps):
            s.update(c=-1.0)
        for _ in range(3):
            s.update(a=-0.3, c=-0.2)
    return g, o


def _positions(size, n, rng, margin=3):
    lo = np.array([-(s // 2) + margin for s in size])
    hi = np.array([s - s // 2 - margin for s in size])
    nodes = rng.integers(lo, hi, (n, len(size))).astype(np.int32)
    real = (nodes + rng.uniform(-0.5, 0.5, nodes.shape)).astype(np.float32)
    return nodes, real


def _oracle_nodes(o, D, p):
    v = o.numeric(tuple(int(x) for x in p))
    return {"grad": v[0:D], "gradF": v[D:2 * D], "gradB": v[2 * D:3 * D],
            "gradC": v[3 * D:4 * D], "gradE": v[4 * D:5 * D], "divergence": v[5 * D],
            "curv": np.float32(o.curv(tuple(int(x) for x in p)))}


def _oracle_real(o, D, p):
    v = o.numeric_f(p)
    return {"grad": v[0:D], "gradF": v[D:2 * D], "gradB": v[2 * D:3 * D],
            "gradC": v[3 * D:4 * D], "gradE": v[4 * D:5 * D], "divergence": v[5 * D],
            "curv": v[5 * D + 1], "get": v[5 * D + 2]}


@pytest.mark.parametrize("size,part,L,steps", [((32, 32, 32), (8, 8, 8), 2, 6),
                                               ((48, 40), (8, 8), 3, 9)])
def test_query_matches_oracle(size, part, L, steps):
    g, o = _both(size, part, L, steps)
    D = len(size)
    nodes, real = _positions(size, 400, np.random.default_rng(21))
    snap = o.snapshot()
    off = np.array(size) // 2
    got = {w: g.query(w, nodes) for w in SCALARS + VECTORS}
    np.testing.assert_array_equal(got["get"], snap[tuple((nodes + off).T)])
    for i, p in enumerate(nodes):
        want = _oracle_nodes(o, D, p)
        for w, v in want.items():
            assert np.array_equal(np.float32(got[w][i]), np.float32(v), equal_nan=True), (w, p)
    got = {w: g.query(w, real) for w in SCALARS + VECTORS}
    for i, p in enumerate(real):
        want = _oracle_real(o, D, p)
        for w, v in want.items():
            assert np.array_equal(np.float32(got[w][i]), np.float32(v), equal_nan=True), (w, p)


def test_query_inside_and_edges():
    fb = _fb()
    g, _ = _both((24, 24, 24), (8, 8, 8), 2, 4)
    pts = np.array([[11.9, 0, 0], [12.0, 0, 0], [-12.0, 0, 0], [-12.01, 0, 0]], np.float32)
    np.testing.assert_array_equal(g.query("inside", pts), [1, 0, 1, 0])
    nodes = np.array([[11, 0, 0], [12, 0, 0], [-12, 0, 0], [-13, 0, 0]], np.int32)
    np.testing.assert_array_equal(g.query("inside", nodes), [1, 0, 1, 0])
    # far outside the grid the isogrid reads as L + 1
    np.testing.assert_array_equal(g.query("get", np.array([[500, 0, 0]], np.int32)), [3.0])
    assert g.query("grad", np.zeros((0, 3), np.float32)).shape == (0, 3)
    with pytest.raises(fb.FeltError):
        g.query(42, np.zeros((1, 3), np.float32))
    with pytest.raises(ValueError):
        g.query("get", np.zeros((2, 2), np.float32))


def test_batch_query_matches_surfaces():
    fb = _fb()
    sizes = [(32, 32, 32), (24, 40, 32)]
    part, L = (8, 8, 8), 2
    b = fb.Batch(sizes, part, L)
    b.seed([(0, 0, 0), (1, -2, 0)])
    os_ = [O.Surface(sz, part, L) for sz in sizes]
    os_[0].seed((0, 0, 0))
    os_[1].seed((1, -2, 0))
    for _ in range(5):
        b.update([dict(c=-1.0), dict(c=-0.8)])
        os_[0].update(c=-1.0)
        os_[1].update(c=-0.8)
    rng = np.random.default_rng(4)
    for i, (o, sz) in enumerate(zip(os_, sizes)):
        _, real = _positions(sz, 200, rng)
        got = b.query(i, "gradE", real)
        for j, p in enumerate(real):
            assert np.array_equal(got[j], _oracle_real(o, 3, p)["gradE"]), (i, p)
        got = b.query(i, "curv", real)
        for j, p in enumerate(real):
            assert np.array_equal(np.float32(got[j]), _oracle_real(o, 3, p)["curv"],
                                  equal_nan=True), (i, p)
