"""fg_snapshot_noalloc: the dense snapshot for callers that cannot allocate device memory while
they run (under another allocator's memory budget, or in a real-time loop that must stay out of
the driver's allocator). It must return exactly what
fg_snapshot returns, on consecutive calls that share its fixed staging array, and reject grids
larger than that array. This file is collected last so that a failure here leaves every other
test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the distance tolerance used by all parity tests; the copies are in fact identical
MAX_FLOATS = 1 << 21


def _snap_noalloc(fb, surf):
    n = int(np.prod(surf.size))
    out = np.full(n, np.nan, dtype=np.float32)
    rc = fb.lib().fg_snapshot_noalloc(surf._h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                      C.c_size_t(n))
    return rc, out.reshape(surf.size)


def test_snapshot_noalloc_matches_snapshot_on_consecutive_calls():
    import felt_b200 as fb
    s = fb.Surface((48, 40, 36), (8, 8, 8), 2)
    s.seed((0, 0, 0))
    for _ in range(5):
        s.update(c=-0.8)
    ref = s.snapshot()
    rc1, a = _snap_noalloc(fb, s)
    rc2, b = _snap_noalloc(fb, s)
    assert rc1 == 0 and rc2 == 0, fb.lib().fg_last_error()
    assert np.abs(a - ref).max() <= TOL
    assert np.abs(b - ref).max() <= TOL
    # the array keeps the last call's contents: a smaller surface after a larger one must
    # still match its own snapshot exactly
    t = fb.Surface((20, 12), (4, 4), 1)
    t.seed((1, 0))
    for _ in range(3):
        t.update(a=-0.3, c=-0.4)
    rc3, c = _snap_noalloc(fb, t)
    assert rc3 == 0
    assert np.abs(c - t.snapshot()).max() <= TOL
    s.update(a=-0.2, c=0.1)
    rc4, d = _snap_noalloc(fb, s)
    assert rc4 == 0
    assert np.abs(d - s.snapshot()).max() <= TOL


def test_snapshot_noalloc_rejects_grids_over_its_limit():
    import felt_b200 as fb
    s = fb.Surface((1500, 1500), (16, 16), 1)  # 2.25M nodes > 2^21
    s.seed((0, 0))
    assert 1500 * 1500 > MAX_FLOATS
    rc, _ = _snap_noalloc(fb, s)
    assert rc == -13  # FG_ERR_CAPACITY
    assert "exceeds" in fb.lib().fg_last_error().decode()
