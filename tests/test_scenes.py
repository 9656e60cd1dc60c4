"""The benchmark scenes that restate a reference fixture: the sphere pile is the reference's sweep's large pile
(core tests, sphere/SphereSweepTest.java:118-144), its jitter drawn from java.util.Random(7) in the fixture's order
(x before z, sphere by sphere); and the oracle steps it through the drop onto the floor."""
import numpy as np

from java_random import JavaRandom
from vxr import scenes
from vxr import spheres as S


def test_the_pile_is_the_reference_fixture():
    side = 16
    sc = scenes.sphere_pile(side=side, seed=7)
    rnd = JavaRandom(7)
    k = 0
    for i in range(side):
        for j in range(side):
            for l_ in range(side):
                assert sc["x"][k] == np.float32(0.07 + 0.06 * i + 0.005 * rnd.next_double())
                assert sc["y"][k] == np.float32(0.3 + 0.07 * j)
                assert sc["z"][k] == np.float32(0.07 + 0.06 * l_ + 0.005 * rnd.next_double())
                k += 1
    assert sc["spheres"] == 4096 and np.all(sc["r"] == np.float32(0.03)) and np.all(sc["im"] == np.float32(10.0))
    assert np.allclose(sc["walls"], (0.08 + 0.06 * side, 0.5 + 0.07 * side, 0.08 + 0.06 * side))
    assert sc["grid"] == S.covering(*sc["walls"], 0.06)


def test_the_oracle_lands_a_small_pile_on_the_floor():
    """A 6^3 pile with the headline solver: after 60 frames it rests on the floor, nothing non-finite."""
    from oracle.sphere import OracleSphereWorld
    sc = scenes.sphere_pile(side=6, seed=7)
    w = OracleSphereWorld(sc["spheres"], sc["substeps"], sc["iterations"], sc["solve"], sc["grid"])
    for k in ("x", "y", "z", "u", "v", "w", "r", "im"):
        w.set_field(k, sc[k])
    w.set_shown(S.shown_at_start(sc["x"], sc["y"], sc["z"], sc["r"]))
    w.set_params(sc["params"], sc["friction"])
    w.step(60)
    y = w.field("y")
    assert np.all(np.isfinite(y)) and np.min(y) >= 0.03 - 1e-3
    assert np.min(y) < 0.031, "the bottom layer is on the floor"
    w.close()
