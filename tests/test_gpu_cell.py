"""The large mixed scene at its configured 1.6 m cell, on the GPU against the oracle: the neighbourhood walk widened
to two cells each way (reach_cells = 2, the 125 cells a narrower-than-rule grid needs; core/box/BoxBroad.java:66-68,
230-252), on 16,384 bodies of the scene's own generator. Candidate pairs bit-exact, and 1 and 20 steps of every state
word and every impulse equal."""
import numpy as np
import pytest

from oracle.box import OracleBoxWorld
from vxr import boxes as B
from vxr import scenes

pytestmark = pytest.mark.gpu

NAMES = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]


@pytest.mark.parametrize("steps", [1, 20])
def test_the_configured_cell_matches_the_oracle(steps):
    from vxr.box_simulation import BoxSimulation
    sc = scenes.sub_volume(262_144, 16_384 / 262_144, seed=8)
    sx, sy, sz = sc["walls"]
    grid = B.covering(sx, sy, sz, 1.6)
    o = OracleBoxWorld(sc["bodies"], sc["substeps"], sc["sweeps"], False, grid, threads=True, reach_cells=2)
    for k in scenes.FIELDS:
        o.set_field(k, sc[k])
    o.set_params(sc["params"])
    g = BoxSimulation(sc["bodies"], sc["substeps"], sc["sweeps"], False, grid, reach_cells=2)
    g.load_state([sc[k] for k in scenes.FIELDS], sc["params"])
    for _ in range(steps):
        assert o.step(1) == tuple(g.step_and_wait(1))
    np.testing.assert_array_equal(g.candidate_pairs(), o.candidate_pairs())
    assert g.touching_pairs() == o.touching_pairs()
    for name, a in zip(NAMES, g.state()):
        assert np.array_equal(a.view(np.int32), o.field(name).view(np.int32)), name
    want = np.array(o.touching_impulses()).reshape(-1, 28)
    assert np.array_equal(g.touching()[4].view(np.int32), want.view(np.int32))
    o.close()
    g.close()
