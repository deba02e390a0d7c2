"""Raycasting on the device (Surface::ray, include/Felt/Surface.hpp:468-616, 1450-1598) against
the reference's own raycasting assertions and, ray for ray, against the CPU oracle.

The device runs the reference's FP32 arithmetic in the same order as the oracle, so hits are
compared bit for bit (misses are FLT_MAX in every component on both sides)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.raycases import FLT_MAX, case_rays, check_case, normalized
from tests.scenario import run_steps

pytestmark = pytest.mark.gpu


def _fb():
    import felt_b200
    return felt_b200


def _golden():
    import json
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "tests", "golden", "reference_golden.json")) as f:
        return json.load(f)["ray"]


def assert_rays_equal(got, want, where=""):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape
    miss_g = np.all(got == np.float32(FLT_MAX), axis=1)
    miss_w = np.all(want == np.float32(FLT_MAX), axis=1)
    bad = np.nonzero(miss_g != miss_w)[0]
    assert bad.size == 0, f"{where}: hit/miss differs for rays {bad[:10]}"
    diff = np.nonzero(np.any(got != want, axis=1))[0]
    assert diff.size == 0, (f"{where}: {diff.size} rays differ, first {diff[0]}: "
                            f"{got[diff[0]]} vs {want[diff[0]]}")


def random_rays(D, size, n, seed):
    """Seeded rays of several kinds: origins inside the grid, origins outside aimed near the
    centre, and axis-aligned directions (zero components exercise the skipped axes)."""
    rng = np.random.default_rng(seed)
    size = np.asarray(size, dtype=np.float64)
    off = -(size // 2)
    k = n // 3
    o_in = off + rng.random((k, D)) * size
    d_in = rng.normal(size=(k, D))
    r = 0.8 * float(size.max())
    u = rng.normal(size=(k, D))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    o_out = u * r
    d_out = -u + 0.25 * rng.normal(size=(k, D))
    m = n - 2 * k
    o_ax = off + rng.random((m, D)) * size
    d_ax = np.zeros((m, D))
    d_ax[np.arange(m), rng.integers(0, D, m)] = rng.choice([-1.0, 1.0], m)
    o = np.concatenate([o_in, o_out, o_ax]).astype(np.float32)
    d = np.concatenate([d_in, d_out, d_ax]).astype(np.float32)
    d = np.array([normalized(v) for v in d], dtype=np.float32)
    return o, d


@pytest.mark.parametrize("case", _golden(), ids=lambda c: c["ref"].split(":")[-1])
def test_ray_golden_device(case):
    fb = _fb()
    g = fb.Surface(case["size"], case["part"], case["layers"])
    o = O.Surface(case["size"], case["part"], case["layers"])
    run_steps(g, case["steps"])
    run_steps(o, case["steps"])
    org, d = case_rays(case)
    hits = g.rays(org, d)
    check_case(case, hits)
    assert_rays_equal(hits, o.rays(org, d), case["ref"])


SCENES = [
    # (size, part, L, seeds, schedule)
    ((48, 48, 48), (8, 8, 8), 2, [(0, 0, 0), (10, 10, 10)],
     [(10, dict(c=-1.0)), (4, dict(a=-0.2, n=0.3, seed=5))]),
    ((40, 40, 40), (5, 5, 5), 3, [(0, 0, 0)], [(12, dict(c=-1.0)), (3, dict(c=0.3))]),
    ((35, 29, 22), (4, 8, 3), 1, [(2, -1, 0)], [(7, dict(c=-0.8, n=0.2, seed=2))]),
    ((64, 64), (4, 4), 2, [(-12, 0), (12, 6)], [(10, dict(c=-1.0)), (5, dict(a=-0.4, c=0.1))]),
    ((33, 47), (3, 5), 4, [(0, 0)], [(8, dict(c=-0.7, n=0.3, seed=9))]),
]


def _scene(scene):
    fb = _fb()
    size, part, L, seeds, schedule = scene
    g = fb.Surface(size, part, L)
    o = O.Surface(size, part, L)
    for s in seeds:
        g.seed(s)
        o.seed(s)
    for n, kw in schedule:
        for _ in range(n):
            g.update(**kw)
            o.update(**kw)
    return g, o


@pytest.mark.parametrize("si", range(len(SCENES)))
def test_ray_random_parity(si):
    g, o = _scene(SCENES[si])
    D = len(SCENES[si][0])
    org, d = random_rays(D, SCENES[si][0], 1500, seed=100 + si)
    hits = g.rays(org, d)
    want = o.rays(org, d)
    assert_rays_equal(hits, want, f"scene {si}")
    hit_frac = float(np.mean(np.any(hits != np.float32(FLT_MAX), axis=1)))
    assert 0.05 < hit_frac < 1.0, hit_frac  # both hits and misses are exercised


@pytest.mark.parametrize("si", range(len(SCENES)))
def test_ray_merge_order_equals_exact_order(si):
    """The kernels order a ray's candidates by merging its per-axis plane walks, from stored
    lists (mode 0) or from cursors (mode 2, the path of rays with long lists); finding each next
    candidate by a full walk (mode 1, the reference's sort restated) gives the same hits."""
    import torch
    g, o = _scene(SCENES[si])
    D = len(SCENES[si][0])
    org, d = random_rays(D, SCENES[si][0], 900, seed=7 + si)
    want = o.rays(org, d)
    to = torch.from_numpy(org).cuda()
    td = torch.from_numpy(d).cuda()
    for mode in (0, 1, 2):
        th = torch.empty_like(to)
        g.rays_device(to.data_ptr(), td.data_ptr(), org.shape[0], th.data_ptr(),
                      order_mode=mode)
        torch.cuda.synchronize()
        assert_rays_equal(th.cpu().numpy(), want, f"order_mode={mode}")


def test_ray_edge_cases():
    fb = _fb()
    g, o = _scene(SCENES[1])
    assert g.rays(np.zeros((0, 3)), np.zeros((0, 3))).shape == (0, 3)
    with pytest.raises(ValueError):
        g.rays(np.zeros((2, 3)), np.zeros((3, 3)))
    with pytest.raises(fb.FeltError):
        g.rays_device(0, 0, 4, 0, order_mode=3)
    # a zero direction never leaves its partition and finds no crossing: a miss on both sides
    org = np.array([[-3.0, 0.5, 0.25], [100.0, 0, 0], [-20.0, -20.0, -20.0]], np.float32)
    d = np.array([[0, 0, 0], [-1, 0, 0], [0, 0, 1]], np.float32)
    assert_rays_equal(g.rays(org, d), o.rays(org, d), "edge rays")
    assert np.all(g.ray(org[0], d[0]) == np.float32(FLT_MAX))


def test_batch_rays_match_single_surfaces():
    fb = _fb()
    sizes = [(32, 32, 32), (40, 24, 32), (24, 24, 24)]
    centres = [(0, 0, 0), (3, -2, 1), (-1, 1, 0)]
    part, L = (8, 8, 8), 2
    b = fb.Batch(sizes, part, L)
    b.seed(centres)
    os_ = [O.Surface(sz, part, L) for sz in sizes]
    for o, c in zip(os_, centres):
        o.seed(c)
    speeds = [dict(c=-1.0), dict(c=-0.7, n=0.3, seed=4), dict(a=-0.3, c=-0.5)]
    for _ in range(6):
        b.update(speeds)
        for o, sp in zip(os_, speeds):
            o.update(**sp)
    for i, (o, sz) in enumerate(zip(os_, sizes)):
        org, d = random_rays(3, sz, 600, seed=40 + i)
        assert_rays_equal(b.rays(i, org, d), o.rays(org, d), f"surface {i}")


def test_ray_convergence_leaving_the_grid_resumes():
    """Where the zero curve meets the grid's walls, some convergences step out of the grid:
    that partition gives ray_miss and the ray goes on with its next candidate (Surface.hpp:
    1491-1494 and 607-614). The device runs those rays in a second pass of its find/converge
    kernels; their hits must still equal the oracle's."""
    fb = _fb()
    scene = ((20, 20, 20), (5, 5, 5), 3, [(0, 0, 0)], [(13, dict(c=-1.0))])
    g, o = _scene(scene)
    org, d = random_rays(3, scene[0], 3000, seed=5)
    l0 = fb.launch_count()
    hits = g.rays(org, d)
    passes = (fb.launch_count() - l0) // 2
    assert passes >= 2, "no convergence left the grid: the scene no longer tests the resume"
    assert_rays_equal(hits, o.rays(org, d), "resumed rays")


def test_ray_long_candidate_lists():
    """Rays crossing many band partitions (three small circles in a row, 2x2 partitions) have
    more candidates than the walk kernel lists per ray and take the cursor path; all three
    candidate orders agree with the oracle."""
    import torch
    scene = ((64, 64), (2, 2), 2, [(-20, 0), (0, 1), (20, -1)], [(3, dict(c=-1.0))])
    g, o = _scene(scene)
    rng = np.random.default_rng(11)
    m = 600
    org = np.stack([np.full(m, -31.5), rng.uniform(-5, 5, m)], axis=1).astype(np.float32)
    d = np.stack([np.ones(m), rng.uniform(-0.05, 0.05, m)], axis=1)
    d = np.array([normalized(v) for v in d.astype(np.float32)], dtype=np.float32)
    want = o.rays(org, d)
    to, td = torch.from_numpy(org).cuda(), torch.from_numpy(d).cuda()
    for mode in (0, 1, 2):
        th = torch.empty_like(to)
        g.rays_device(to.data_ptr(), td.data_ptr(), m, th.data_ptr(), order_mode=mode)
        torch.cuda.synchronize()
        assert_rays_equal(th.cpu().numpy(), want, f"order_mode={mode}")
