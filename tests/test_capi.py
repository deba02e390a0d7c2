"""CPU checks of the drop-in boundary: the C-ABI library loads and exports every symbol that
include/felt_gpu.h declares (no compute without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "felt_gpu.h")).read()
    return sorted(set(re.findall(r"FG_API\s+(?:const\s+char\s*\*|int)\s+(fg_\w+)\s*\(", hdr)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fg_surface_create" in syms and "fg_update_builtin" in syms and "fg_polys_march" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol():
    path = os.path.join(ROOT, "felt_b200", "libfelt_gpu.so")
    if not os.path.exists(path):
        import felt_b200
        felt_b200.build()
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_create_without_device_fails_cleanly():
    """With no CUDA device the engine reports an error code instead of crashing or falling
    back to the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import felt_b200
    with pytest.raises(felt_b200.FeltError) as ei:
        felt_b200.Surface((16, 16), (8, 8), 2)
    assert ei.value.code == -2
