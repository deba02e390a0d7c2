"""Ray inputs and checks of the reference's raycasting tests (src/tests/test_Surface.cpp:1284-1442,
1479-1533), shared by the oracle and device tests.

The rotation sweeps build their rays with Eigen's AngleAxisf(angle, axis).matrix() (Eigen 3,
AngleAxis::toRotationMatrix, the Rodrigues formula) in float32: rot_mult runs 0, 0.1, ... while
below 2 (accumulated in float32), origin = R (0, 0, -10), dir = normalized(R (0, 0, 1)). The
reference only asserts that every such ray hits; the hit points need no bit-level agreement with
Eigen, only the same rays for the oracle and the device."""
import numpy as np

F = np.float32
FLT_MAX = float(np.finfo(np.float32).max)


def normalized(v):
    """Eigen normalized(): v / sqrt(x0^2 + (x1^2 + x2^2)) in float32."""
    v = np.asarray(v, dtype=F)
    sq = v * v
    z = sq[0] + (sq[1] + sq[2]) if len(v) == 3 else sq[0] + sq[1]
    return v / np.sqrt(F(z)) if z > 0 else v


def rotation(angle, axis):
    """Eigen AngleAxis::toRotationMatrix in float32."""
    a = np.asarray(axis, dtype=F)
    s, c = np.sin(F(angle)), np.cos(F(angle))
    sa = s * a
    ca = (F(1) - c) * a
    r = np.zeros((3, 3), dtype=F)
    t = ca[0] * a[1]
    r[0, 1], r[1, 0] = t - sa[2], t + sa[2]
    t = ca[0] * a[2]
    r[0, 2], r[2, 0] = t + sa[1], t - sa[1]
    t = ca[1] * a[2]
    r[1, 2], r[2, 1] = t - sa[0], t + sa[0]
    for i in range(3):
        r[i, i] = ca[i] * a[i] + c
    return r


def sweep_rays(axis, normalize_axis):
    """The (origins, dirs) of one rotation sweep (test_Surface.cpp:1378-1398)."""
    ax = normalized(axis) if normalize_axis else np.asarray(axis, dtype=F)
    org, dirs = [], []
    rot_mult = F(0)
    while rot_mult < F(2.0):
        r = rotation(rot_mult * F(np.pi), ax)
        org.append(r @ np.array([0, 0, -10], dtype=F))
        dirs.append(normalized(r @ np.array([0, 0, 1], dtype=F)))
        rot_mult = F(rot_mult + F(0.1))
    return np.array(org, dtype=F), np.array(dirs, dtype=F)


def case_rays(case):
    """(origins, dirs) of a golden ray case: one ray, or a rotation sweep."""
    if "sweep_axis" in case:
        return sweep_rays(case["sweep_axis"], case["normalize_axis"])
    d = np.asarray(case["dir"], dtype=F)
    if case["normalize"]:
        d = normalized(d)
    return np.array([case["origin"]], dtype=F), d[None, :]


def is_miss(hit):
    """Surface::ray_miss: FLT_MAX in every component."""
    return bool(np.all(np.asarray(hit) == F(FLT_MAX)))


def approx_vec(got, want, eps=None):
    """ApproxVec (src/tests/Utils.hpp:64-131): per component
    |a - b| < eps * (1 + max(|a|, |b|)), eps = 100 * FLT_EPSILON unless given."""
    eps = float(np.finfo(np.float32).eps) * 100 if eps is None else eps
    g = np.asarray(got, dtype=np.float64)
    w = np.asarray(want, dtype=np.float64)
    return bool(np.all(np.abs(g - w) < eps * (1.0 + np.maximum(np.abs(g), np.abs(w)))))


def check_case(case, hits):
    """The reference's assertion for a golden ray case, on the hits of case_rays(case)."""
    if case["expect"] == "miss":
        assert all(is_miss(h) for h in hits), hits
    elif case["expect"] == "hit":
        bad = [i for i, h in enumerate(hits) if is_miss(h)]
        assert not bad, f"rays {bad} missed"
    else:
        assert len(hits) == 1
        assert approx_vec(hits[0], case["hit"], case["epsilon"]), (hits[0], case["hit"])
