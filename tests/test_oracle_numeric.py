"""The Numeric API at real positions in the oracle (NumericMixin.hpp:72-481 with a float
position type): at whole-number positions it reads the nodes themselves (interp's fractions
are 0), so it equals the node version; on a field that is linear over the cells it reads, the
interpolated value and the gradients take their closed forms."""
import numpy as np
import pytest

from oracle import oracle as O


def _grown(size, part, L, steps):
    s = O.Surface(size, part, L)
    s.seed(tuple(0 for _ in size))
    for _ in range(steps):
        s.update(c=-1.0)
    for _ in range(2):
        s.update(a=-0.3, c=-0.2)
    return s


@pytest.mark.parametrize("size,part,L", [((32, 32, 32), (8, 8, 8), 2), ((40, 36), (6, 6), 3)])
def test_whole_positions_equal_the_node_version(size, part, L):
    s = _grown(size, part, L, 5)
    D = len(size)
    rng = np.random.default_rng(3)
    lo = np.array([-(n // 2) + 2 for n in size])
    hi = np.array([n - n // 2 - 3 for n in size])
    for _ in range(200):
        p = tuple(int(x) for x in rng.integers(lo, hi))
        got = s.numeric_f(p)
        assert np.array_equal(got[:5 * D + 1], s.numeric(p)), p
        # curv is 0/0 = NaN where every sample is background, on both sides
        assert np.array_equal(got[5 * D + 1:5 * D + 2], np.float32([s.curv(p)]), equal_nan=True), p
        assert got[5 * D + 2] == s.snapshot()[tuple(np.array(p) + np.array(size) // 2)], p


def test_linear_field_closed_form():
    """A seed at the origin leaves phi = |x| + |y| + |z| on the band nodes (L = 3) and the
    background L + 1 = 4 beyond them, so every cell within city-block distance 4 of the origin
    holds phi = |x| + |y| + |z|, which is linear on each cell, and the interpolation
    reproduces it. At p = (0.3, 0.2, 0.45) the samples p +- e_a all lie in such cells."""
    s = O.Surface((24, 24, 24), (8, 8, 8), 3)
    s.seed((0, 0, 0))
    p = np.array([0.3, 0.2, 0.45])
    v = s.numeric_f(tuple(p))
    tol = 1e-5
    phi = lambda q: float(np.abs(q).sum())  # noqa: E731
    e = np.eye(3)
    fwd = np.array([phi(p + e[a]) for a in range(3)])
    back = np.array([phi(p - e[a]) for a in range(3)])
    c = phi(p)
    np.testing.assert_allclose(v[0:3], (fwd - back) / 2, atol=tol)  # grad
    np.testing.assert_allclose(v[3:6], fwd - c, atol=tol)  # gradF
    np.testing.assert_allclose(v[6:9], c - back, atol=tol)  # gradB
    np.testing.assert_allclose(v[9:12], (fwd - back) / 2, atol=tol)  # gradC
    np.testing.assert_allclose(v[12:15], np.maximum(c - back, 0) + np.minimum(fwd - c, 0),
                               atol=tol)  # gradE
    np.testing.assert_allclose(v[15], ((fwd - c) - (c - back)).sum(), atol=tol)  # divergence
    np.testing.assert_allclose(v[17], c, atol=tol)  # interp
    assert np.isfinite(v[16])  # curv


def test_each_function_steps_its_own_position():
    """gradF steps +1, -1 per axis, gradB -1, +1, gradC -1, +2, -1 (NumericMixin.hpp:279-355),
    each on its own copy of the position; in float the undo need not restore the coordinate,
    and the drift carries into the next axis. Restated here in numpy float32 over the oracle's
    interp (the last value numeric_f returns)."""
    s = _grown((32, 32, 32), (8, 8, 8), 2, 6)
    f32 = np.float32
    interp = lambda q: s.numeric_f(q)[17]  # noqa: E731
    rng = np.random.default_rng(8)
    for _ in range(60):
        q = (rng.integers(-8, 8, 3) + rng.uniform(-0.5, 0.5, 3)).astype(np.float32)
        v = s.numeric_f(q)
        c = interp(q)
        t = q.copy()
        gf = np.zeros(3, np.float32)
        for a in range(3):
            t[a] = f32(t[a] + f32(1))
            gf[a] = f32(interp(t) - c)
            t[a] = f32(t[a] - f32(1))
        t = q.copy()
        gb = np.zeros(3, np.float32)
        for a in range(3):
            t[a] = f32(t[a] - f32(1))
            gb[a] = f32(c - interp(t))
            t[a] = f32(t[a] + f32(1))
        t = q.copy()
        gc = np.zeros(3, np.float32)
        for a in range(3):
            t[a] = f32(t[a] - f32(1))
            b = interp(t)
            t[a] = f32(t[a] + f32(2))
            fw = interp(t)
            t[a] = f32(t[a] - f32(1))
            gc[a] = f32(f32(fw - b) / f32(2))
        assert np.array_equal(v[3:6], gf), (q, v[3:6], gf)
        assert np.array_equal(v[6:9], gb), (q, v[6:9], gb)
        assert np.array_equal(v[9:12], gc), (q, v[9:12], gc)
