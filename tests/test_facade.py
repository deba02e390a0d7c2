"""The C++ facade (felt_b200/include/felt_gpu/surface.hpp + device.cuh): a program written the
way a user of the reference writes one, with its own __device__ speed functors in each of the
reference's three functor signatures, compiled by nvcc against libfelt_gpu.so. On the GPU its
result equals the oracle's run of the same speeds."""
import os
import subprocess

import numpy as np
import pytest

from tests.dumps import first_difference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = "/usr/local/cuda/bin/nvcc"
LIB_DIR = os.path.join(ROOT, "felt_b200")
SRC = os.path.join(ROOT, "felt_b200", "examples", "custom_speed.cu")


def _compile(out, link):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "-fmad=false", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "felt_b200", "include"), SRC]
    if link:
        if not os.path.exists(os.path.join(LIB_DIR, "libfelt_gpu.so")):
            pytest.fail("libfelt_gpu.so is not built (run __graft_entry__.build())")
        cmd += ["-L", LIB_DIR, "-lfelt_gpu", "-Xlinker", "-rpath," + LIB_DIR, "-o", out]
    else:
        cmd += ["-c", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_facade_compiles_with_device_functors(tmp_path):
    _compile(str(tmp_path / "custom_speed.o"), link=False)


@pytest.mark.gpu
def test_device_functors_match_oracle(tmp_path):
    from oracle import oracle as O
    exe = str(tmp_path / "custom_speed")
    _compile(exe, link=True)
    pre = str(tmp_path / "out")
    r = subprocess.run([exe, pre], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dump = np.fromfile(pre + ".dump", dtype=np.uint32)
    phi = np.fromfile(pre + ".phi", dtype=np.float32)
    o = O.Surface((32, 32, 32), (8, 8, 8), 2)
    o.seed((0, 0, 0))
    for _ in range(12):
        o.update(a=-0.3, c=-0.2)
    for _ in range(4):
        o.update(n=0.1, seed=7, c=-0.25)
    for _ in range(2):
        o.update(c=0.2)
    d = first_difference(dump, o.dump())
    assert d is None, d
    assert float(np.abs(phi - o.snapshot().reshape(-1)).max()) <= 1e-5


PROBE = os.path.join(ROOT, "felt_b200", "examples", "numeric_probe.cu")


def _compile_probe(out, link):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "-fmad=false", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "felt_b200", "include"), PROBE]
    if link:
        cmd += ["-L", LIB_DIR, "-lfelt_gpu", "-Xlinker", "-rpath," + LIB_DIR, "-o", out]
    else:
        cmd += ["-c", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_numeric_probe_compiles(tmp_path):
    _compile_probe(str(tmp_path / "numeric_probe.o"), link=False)


@pytest.mark.gpu
def test_numeric_api_matches_oracle(tmp_path):
    """grad, gradF, gradB, gradC, gradE and divergence (NumericMixin.hpp:165-355) called from a
    __device__ functor at every zero-layer node, and the same with curv and interp at the real
    position node + (0.3, -0.2, 0.45), equal the oracle's, bit for bit."""
    from oracle import oracle as O
    exe = str(tmp_path / "numeric_probe")
    _compile_probe(exe, link=True)
    out = str(tmp_path / "numeric.bin")
    r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n = 32
    vals = np.fromfile(out, dtype=np.float32).reshape(n, n, n, 35)
    o = O.Surface((n, n, n), (8, 8, 8), 2)
    o.seed((0, 0, 0))
    for _ in range(6):
        o.update(c=-1.0)
    for _ in range(4):
        o.update(a=-0.3, c=-0.2)
    idx = np.argwhere(vals[..., 16] == 1.0)
    assert len(idx) > 100
    assert len(idx) == o.layer_size(0)
    for i, j, k in idx:
        pos = (int(i) - n // 2, int(j) - n // 2, int(k) - n // 2)
        want = o.numeric(pos)
        got = vals[i, j, k, :16]
        assert np.array_equal(got, want), (pos, got, want)
        q = np.float32(pos) + np.float32([0.3, -0.2, 0.45])
        want_f = o.numeric_f(q)
        got_f = vals[i, j, k, 17:]
        assert np.array_equal(got_f, want_f, equal_nan=True), (tuple(q), got_f, want_f)
