"""The broad phase with no allocation (vxr_box_broadphase_static), for callers that cannot allocate device memory
while stepping: a host that owns all device memory through its own pool, or code that must not allocate between
the launches it records or under a frame deadline. Its scratch is a fixed array in the library; the caller brings
the inputs and outputs (here torch tensors stand in for the caller's own memory).

Checked against the existing entry point: the candidate pairs a world's step lists (vxr_box_candidates) from the
same state, which must be the same sorted pairs exactly (integer output, so the tolerance is equality), on two
calls in a row of different sizes, the second after the first has left its contents in the shared scratch. Kept in
a file of its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest

from vxr import boxes as B
from vxr import _lib

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "z", "qx", "qy", "qz", "qw", "hx", "hy", "hz", "shape"]


def world_candidates(scene):
    """Candidate pairs of one step of a world started from `scene` (the existing entry point)."""
    from vxr.box_simulation import BoxSimulation
    w = BoxSimulation(scene["bodies"], 1, 1, False, scene["grid"])
    l = [scene["lx"], scene["ly"], scene["lz"]]
    q = [scene["qx"], scene["qy"], scene["qz"], scene["qw"]]
    h = [scene["hx"], scene["hy"], scene["hz"]]
    w.start_momentum(scene["x"], scene["y"], scene["z"], scene["u"], scene["v"], scene["w"], l, q, h,
                     scene["shape"], scene["im"], scene["params"])
    w.step(1)
    pairs = w.candidate_pairs()
    w.close()
    return pairs


def static_candidates(scene, capacity=None):
    import torch
    dev = torch.device("cuda:0")
    n = scene["bodies"]
    fields = [torch.from_numpy(np.ascontiguousarray(scene[k], np.float32)).to(dev) for k in FIELDS]
    capacity = capacity if capacity is not None else n * B.SLOTS
    first = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device=dev)
    second = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device=dev)
    result = torch.zeros(3, dtype=torch.int32, device=dev)
    ptrs = (ctypes.c_void_p * 11)(*[t.data_ptr() for t in fields])
    g = scene["grid"]
    stream = torch.cuda.current_stream(dev)
    rc = _lib.lib().vxr_box_broadphase_static(n, ptrs, _lib.Grid(g.nx, g.ny, g.nz, g.cell), 1,
                                              float(B.bits_f32(scene["params"][B.MARGIN])), ctypes.c_void_p(
                                                  first.data_ptr()), ctypes.c_void_p(second.data_ptr()), capacity,
                                              ctypes.c_void_p(result.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    torch.cuda.synchronize()
    found, unlisted, status = [int(v) for v in result.cpu()]
    kept = min(found, capacity)
    return np.stack([first[:kept].cpu().numpy(), second[:kept].cpu().numpy()], axis=1), found, status


def broad_scene():
    import box_cases as C
    sc = C.broad_fixture()
    grid = B.grid(sc.sx, sc.sy, sc.sz, sc.widest, sc.margin)
    d = {k: getattr(sc, k) for k in ("x", "y", "z", "u", "v", "w")}
    d.update({"lx": sc.l[0], "ly": sc.l[1], "lz": sc.l[2], "qx": sc.q[0], "qy": sc.q[1], "qz": sc.q[2],
              "qw": sc.q[3], "hx": sc.half[0], "hy": sc.half[1], "hz": sc.half[2], "shape": sc.shape, "im": sc.im,
              "bodies": sc.n, "grid": grid, "params": sc.param_bits()})
    return d


def test_static_broad_phase_matches_the_world_twice_in_a_row():
    from vxr import scenes
    first_scene = scenes.sub_volume(262_144, 4096 / 262_144, seed=5)
    second_scene = broad_scene()
    for scene in (first_scene, second_scene):
        got, found, status = static_candidates(scene)
        want = world_candidates(scene)
        assert status == 0
        assert found == len(want)
        np.testing.assert_array_equal(got, want)


def test_static_broad_phase_reports_a_short_output():
    scene = broad_scene()
    want = world_candidates(scene)
    got, found, status = static_candidates(scene, capacity=10)
    assert status == _lib.VXR_ECAPACITY and found == len(want)
    np.testing.assert_array_equal(got, want[:10])


def test_static_broad_phase_rejects_sizes_beyond_its_scratch():
    g = _lib.Grid(4, 4, 4, 1.0)
    dummy = (ctypes.c_void_p * 11)(*([1] * 11))  # never read: the sizes are refused first
    rc = _lib.lib().vxr_box_broadphase_static(16385, dummy, g, 1, 0.0, ctypes.c_void_p(1), ctypes.c_void_p(1), 0,
                                              ctypes.c_void_p(1), None)
    assert rc == _lib.VXR_ECAPACITY
    big = _lib.Grid(100, 100, 100, 1.0)
    rc = _lib.lib().vxr_box_broadphase_static(8, dummy, big, 1, 0.0, ctypes.c_void_p(1), ctypes.c_void_p(1), 0,
                                              ctypes.c_void_p(1), None)
    assert rc == _lib.VXR_ECAPACITY
