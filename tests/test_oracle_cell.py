"""The large mixed scene's configured 1.6 m cell. The reference's rule (core/box/BoxBroad.java:66-68) needs cells as
wide as the widest bounding sphere plus the margin, about 2.08 m for this scene (boxes reach 1.04 m from their
centres), because its walk (around, :230-252) visits only the 27 cells about a body's own. A 1.6 m grid keeps every
pair when the walk widens to two cells each way (125 cells). On the oracle: the widened walk over 1.6 m cells lists
exactly the candidate pairs of the reference's rule grid, and the steps that follow are the same to the bit."""
import numpy as np

from oracle.box import OracleBoxWorld
from vxr import boxes as B
from vxr import scenes

NAMES = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]


def oracle(sc, grid, reach):
    o = OracleBoxWorld(sc["bodies"], sc["substeps"], sc["sweeps"], False, grid, threads=True, reach_cells=reach)
    for k in scenes.FIELDS:
        o.set_field(k, sc[k])
    o.set_params(sc["params"])
    return o


def test_a_narrow_grid_with_a_wider_walk_lists_the_rule_grids_pairs():
    sc = scenes.sub_volume(262_144, 4096 / 262_144, seed=6)
    sx, sy, sz = sc["walls"]
    narrow = B.covering(sx, sy, sz, 1.6)
    assert narrow.cell < sc["grid"].cell  # the configured cell is below the rule's
    rule = oracle(sc, sc["grid"], 1)
    wide = oracle(sc, narrow, 2)
    for _ in range(3):
        a = rule.step(1)
        b = wide.step(1)
        assert a == b and a[4] == 0  # the same report, nothing unlisted
        np.testing.assert_array_equal(wide.candidate_pairs(), rule.candidate_pairs())
    for k in NAMES:
        assert np.array_equal(wide.field(k).view(np.int32), rule.field(k).view(np.int32)), k
    rule.close()
    wide.close()
