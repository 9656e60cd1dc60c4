"""Failure paths of the step, made to happen without faulting or hanging the GPU: every case is a bounded device
wait made short, a capacity made small, a round limit made low, or a bad value on the host. After each, the same
GPU steps a scene again and matches the oracle to the bit, so the context stayed usable.

The reference's counterparts: IllegalStateException for a pass that never ends
(core/sphere/SphereStepper.java:79,86-88, tested at ctest/sphere/SphereStepperTest.java:163-166), the broken flag for
non-finite state (core/sphere/SphereDiagnostics.java:48-50), IllegalArgumentException for sizes
(core/box/BoxStep.java:82-85).
"""
import numpy as np
import pytest

import box_cases as C
import sphere_cases as SC
from vxr import _lib, scenes
from vxr._lib import VxrError

pytestmark = pytest.mark.gpu


def still_matches_the_oracle(steps=5):
    """A mixed pile stepped on the GPU and on the oracle: every state word equal."""
    a = C.mixed_pile_scene()
    b = C.mixed_pile_scene()
    a.start("oracle")
    b.start("gpu")
    for _ in range(steps):
        assert tuple(a.world.step(1)) == tuple(b.world.step(1))
    a.read()
    b.read()
    for fa, fb in zip([a.x, a.y, a.z, a.u, a.v, a.w, a.l, a.q], [b.x, b.y, b.z, b.u, b.v, b.w, b.l, b.q]):
        np.testing.assert_array_equal(fb, fa)
    a.close()
    b.close()


def pile_world():
    s = C.pile_scene(7)
    s.start("gpu")
    return s


def test_a_grid_wait_that_runs_out_stops_the_step_with_a_timeout():
    """A wait limit of one nanosecond: the first grid barrier a block must wait at gives up, raises the abort word,
    and every block leaves at its next barrier. The step returns VXR_ETIMEOUT; the world steps again once the limit
    is back and a state is loaded."""
    s = pile_world()
    s.world.step(2)
    s.world.wait_limit(1)
    with pytest.raises(VxrError) as err:
        s.world.step(1)
    assert err.value.status == _lib.VXR_ETIMEOUT
    s.world.wait_limit(0)
    fresh = C.pile_scene(7)
    fresh.start("gpu")
    ref = fresh.world
    s.world.start_momentum(fresh.x, fresh.y, fresh.z, fresh.u, fresh.v, fresh.w, fresh.l, fresh.q, fresh.half,
                           fresh.shape, fresh.im, fresh.param_bits())
    for _ in range(3):
        assert tuple(s.world.step(1)) == tuple(ref.step(1))
    for x, y in zip(s.world.state(), ref.state()):
        np.testing.assert_array_equal(x, y)
    ref.close()
    s.close()
    still_matches_the_oracle()


def test_more_candidate_pairs_than_the_capacity_is_reported():
    """A world made with room for 16 candidate pairs over a pile that has hundreds: the step keeps to the room it
    has and returns VXR_ECAPACITY."""
    from vxr.box_simulation import BoxSimulation
    s = C.pile_scene(7)
    s.start("gpu")
    small = BoxSimulation(s.n, s.substeps, s.passes, False, s.grid, max_pairs=16)
    small.start_momentum(s.x, s.y, s.z, s.u, s.v, s.w, s.l, s.q, s.half, s.shape, s.im, s.param_bits())
    with pytest.raises(VxrError) as err:
        small.step(1)
    assert err.value.status == _lib.VXR_ECAPACITY
    small.close()
    s.close()
    still_matches_the_oracle()


def test_a_pass_still_open_past_the_round_limit_is_an_error_not_a_hang():
    """The crowded until-done pile with the round limit at one round: a pass that needs more rounds than its
    opening batch stops the step with VXR_EROUNDS; the default limit steps the same scene."""
    s = SC.until_done_pile()
    s.start("gpu")
    s.world.round_limit(1)
    with pytest.raises(VxrError) as err:
        for _ in range(5):
            s.world.step_and_wait(1)
    assert err.value.status == _lib.VXR_EROUNDS
    s.close()
    ok = SC.until_done_pile()
    ok.start("gpu")
    ok.advance(3)
    ok.close()
    still_matches_the_oracle()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_a_non_finite_state_is_refused(bad):
    """A NaN or an infinity in a state to load: VXR_ENONFINITE and nothing loaded (the world keeps stepping the
    state it had)."""
    sc = scenes.sub_volume(262_144, 512 / 262_144, seed=2)
    from vxr.box_simulation import BoxSimulation
    w = BoxSimulation(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"])
    fields = [sc[k].copy() for k in scenes.FIELDS]
    w.load_state(fields, sc["params"])
    w.step_and_wait(2)
    before = w.state()
    broken = [f.copy() for f in fields]
    broken[4][7] = bad  # v of body 7
    with pytest.raises(VxrError) as err:
        w.load_state(broken, sc["params"])
    assert err.value.status == _lib.VXR_ENONFINITE
    for x, y in zip(w.state(), before):
        np.testing.assert_array_equal(x, y)
    w.step_and_wait(1)
    w.close()

    sp = SC.until_done_pile()
    sp.start("gpu")
    r = sp.r.copy()
    r[3] = bad
    with pytest.raises(VxrError) as err:
        sp.world.start(sp.x, sp.y, sp.z, sp.u, sp.v, sp.w, r, sp.im, sp.param_bits())
    assert err.value.status == _lib.VXR_ENONFINITE
    sp.close()
