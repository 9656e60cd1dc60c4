"""The C-ABI library loads, exports every symbol include/vxr.h declares, and its host-only helpers agree with
the Python mirror of the reference's host code (no GPU needed)."""
import os
import re

import numpy as np
import pytest

from vxr import _lib, boxes as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "vxr.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(vxr_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(_lib.SYMBOLS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert b"sm_100a" in L.vxr_version()


@pytest.mark.parametrize("args", [
    (1 / 600, 0, -9.81, 0, 1, 1, 1, 0, 0, 0.005, 0),
    (1 / 480, 0.3, -9.8, 0.1, 128, 70, 128, 0.5, 0.5, 0.005, 0.1),
    (1e-3, 0, 0, 0, 1, 1, 1, 0, 0, 0.01, 0),
    (1 / 120, 0, -9.81, 0, 20, 40, 20, 0.6, 0.6, 0.0, 0.3),
])
def test_params_match_the_reference_host_code(args):
    from vxr.box_simulation import make_params
    assert list(make_params(*args)) == B.params(*args)


def test_params_reject_what_the_reference_rejects():
    from vxr.box_simulation import make_params
    from vxr._lib import VxrError
    for bad in [(0, 0, 0, 0, 1, 1, 1), (1e-3, 0, 0, 0, 0, 1, 1), (1e-3, 0, 0, 0, 1, 1, 1, -1)]:
        with pytest.raises(ValueError):
            B.params(*bad)
        with pytest.raises(VxrError):
            make_params(*bad)


def test_grid_matches_the_reference_rule():
    g = _lib.Grid()
    L = _lib.lib()
    assert L.vxr_box_make_grid(128.0, 70.0, 128.0, 1.0392304845, 0.005, g) == 0
    ref = B.grid(128.0, 70.0, 128.0, 1.0392304845, 0.005)
    assert (g.nx, g.ny, g.nz) == (ref.nx, ref.ny, ref.nz)
    assert np.float32(g.cell) == np.float32(ref.cell)


def test_static_broad_phase_refuses_a_reach_beyond_the_grid():
    """vxr_box_broadphase_static refuses a negative reach or one wider than the grid's widest side before it touches
    a device: an unbounded reach would only lengthen every thread's neighbourhood walk."""
    import ctypes
    L = _lib.lib()
    g = _lib.Grid(4, 6, 5, 1.0)
    dummy = (ctypes.c_void_p * 11)(*([1] * 11))  # never read: the arguments are refused first
    one = ctypes.c_void_p(1)
    for reach in (-1, 7, 645, 1 << 30):
        assert L.vxr_box_broadphase_static(8, dummy, g, reach, 0.0, one, one, 0, one, None) == _lib.VXR_EINVAL


def test_measurement_entry_points_refuse_a_missing_world():
    """The measurement calls (given starts, first substeps, the residual's parts, the list kernel, the island switch)
    answer a null world with VXR_EINVAL before they touch a device."""
    L = _lib.lib()
    assert L.vxr_box_first_substeps(None, 1, 1) == _lib.VXR_EINVAL
    assert L.vxr_box_learned_given(None, None, 0, 1) == _lib.VXR_EINVAL
    assert L.vxr_box_residual_parts(None, None, None, 0) == -_lib.VXR_EINVAL
    assert L.vxr_box_residuals(None, None, 0, None) == -_lib.VXR_EINVAL
    assert L.vxr_box_learned(None, None, 0) == _lib.VXR_EINVAL
