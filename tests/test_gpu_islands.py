"""Islands: the small connected components of a step's placed touching pairs solved whole by one thread block each
(and bodies in no placed pair by a thread each), apart from the grid-wide phases that the larger components go through.

The reference's order of operations is a per-body order (core/box/BoxStep.java:199-231: each sweep every round,
then the walls), and bodies of different components share no pair, so the schedule changes no result. Checked to the
bit: the large mixed scene's own generator on a 16,384-body part of its volume, stepped with islands and without,
through the drop (small islands in the air, lone bodies on the floor and at the walls); a crowded drop in which a
pile larger than a block's component forms beside small islands; and against the oracle over the first steps.
"""
import numpy as np
import pytest

from vxr import scenes

pytestmark = pytest.mark.gpu

NAMES = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]


def gpu_world(sc, islands=True):
    from vxr.box_simulation import BoxSimulation
    w = BoxSimulation(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"])
    w.load_state([sc[k] for k in scenes.FIELDS], sc["params"])
    w.islands(islands)
    return w


def oracle_world(sc):
    from oracle.box import OracleBoxWorld
    o = OracleBoxWorld(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"], threads=True)
    for k in scenes.FIELDS:
        o.set_field(k, sc[k])
    o.set_params(sc["params"])
    return o


def assert_same_state(got, want, what):
    for name, a, b in zip(NAMES, got, want):
        assert np.array_equal(np.asarray(a).view(np.int32), np.asarray(b).view(np.int32)), f"{what}: {name}"


def assert_same_worlds(a, b, what):
    assert_same_state(a.state(), b.state(), what)
    for x, y in zip(a.touching(), b.touching()):
        assert np.array_equal(np.asarray(x).view(np.int32), np.asarray(y).view(np.int32)), what
    for x, y in zip(a.walls(), b.walls()):
        assert np.array_equal(x.view(np.int32), y.view(np.int32)), what


def test_islands_and_grid_phases_agree_through_the_drop():
    """150 steps of a 16,384-body part of the large mixed scene, with islands and without: every state word, every
    pair impulse and every wall record equal after every 25 steps."""
    sc = scenes.sub_volume(262_144, 16_384 / 262_144, seed=3)
    a = gpu_world(sc, islands=True)
    b = gpu_world(sc, islands=False)
    seen = {"islands": 0, "alone": 0}
    for k in range(6):
        ra = a.step_and_wait(25)
        rb = b.step_and_wait(25)
        assert tuple(ra) == tuple(rb)
        p = a.paths()
        seen["islands"] += p["islands"]
        seen["alone"] += p["alone"]
        assert b.paths()["grid"] == sc["bodies"]
        assert_same_worlds(a, b, f"after {25 * (k + 1)} steps")
    assert seen["islands"] > 0 and seen["alone"] > 0
    a.close()
    b.close()


def test_a_pile_larger_than_a_block_sends_every_body_to_the_grid_phases():
    """A crowded drop into a low box: once a component larger than a block's forms, every body of the step takes the
    grid phases (their phase count is set by the rounds alone); before, the components take island blocks. Equal to
    the bit throughout."""
    sc = scenes.large_mixed(4096, seed=9, volume=(24.0, 6.0, 24.0), height=12.0)
    a = gpu_world(sc, islands=True)
    b = gpu_world(sc, islands=False)
    seen = set()
    for k in range(8):
        a.step_and_wait(1 if k < 4 else 15)
        b.step_and_wait(1 if k < 4 else 15)
        p = a.paths()
        if p["largest"] > 256:
            assert p["grid"] == sc["bodies"] and p["islands"] == 0 and p["alone"] == 0
            seen.add("grid")
        else:
            seen.add("islands")
        assert_same_worlds(a, b, f"after check {k}")
    assert "grid" in seen
    a.close()
    b.close()


@pytest.mark.parametrize("steps", [1, 20])
def test_the_large_scene_generator_matches_the_oracle(steps):
    """16,384 bodies of the large mixed scene's distribution (its body density, shapes and sizes), 1 and 20 steps:
    candidate pairs, touching pairs, impulses and every state word equal to the oracle's."""
    sc = scenes.sub_volume(262_144, 16_384 / 262_144, seed=4)
    o = oracle_world(sc)
    g = gpu_world(sc)
    for _ in range(steps):
        ro = o.step(1)
        rg = g.step_and_wait(1)
        assert ro == tuple(rg)[:5]
    np.testing.assert_array_equal(g.candidate_pairs(), o.candidate_pairs())
    assert g.touching_pairs() == o.touching_pairs()
    assert_same_state(g.state(), [o.field(k) for k in NAMES], f"after {steps} steps")
    want = np.array(o.touching_impulses()).reshape(-1, 28)
    got = g.touching()[4]
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    o.close()
    g.close()
