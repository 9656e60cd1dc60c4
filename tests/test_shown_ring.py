"""The picture's hand-off ring: the reference's ShownRingTest (vexelray-sim-rigid-gui/src/test/java/dev/vexelray/sim/
rigid/gui/ShownRingTest.java:22-94), run against the native ring with no device (generations of no bodies keep no
buffers); and, on the GPU, frames that carry the steps' pictures."""
import numpy as np
import pytest

from vxr.shown_ring import SPHERES, ShownRing


def ring():
    return ShownRing()


def test_nothing_is_taken_before_a_step_is_published():
    r = ring()
    r.install(SPHERES, 0)
    assert r.take() is None
    r.close()


def test_the_writer_never_keeps_a_step_where_the_frame_reads_or_has_been_offered():
    r = ring()
    r.install(SPHERES, 0)
    front = None
    for step in range(1, 201):
        back = r.back()
        if front is not None:
            assert front.slot != back, f"step {step} would be kept in the slot the frame reads"
        r.publish(step, step * 1_000_000)
        assert back != r.back(), "nor in the slot just offered"
        if step % 3 == 0 or step % 7 == 0:
            front = r.take()
            assert front.step == step, "the frame takes the newest finished step"
    r.close()


def test_a_frame_with_nothing_new_keeps_what_it_has():
    r = ring()
    r.install(SPHERES, 0)
    r.publish(1, 1)
    first = r.take()
    again = r.take()
    assert (first.generation, first.slot, first.step) == (again.generation, again.slot, again.step)
    r.close()


def test_an_old_generation_is_retired_only_once_the_frame_has_moved_past_it():
    r = ring()
    one = r.install(SPHERES, 0)
    r.publish(1, 1)
    r.take()
    two = r.install(SPHERES, 0)
    r.publish(1, 2)
    assert r.retired() == [], "the frame still reads the first generation's slot"
    assert r.take().generation == two
    assert r.retired() == [one]
    assert r.retired() == [], "each once"
    r.close()


def test_a_generation_the_frame_never_took_is_retired_at_the_next():
    r = ring()
    one = r.install(SPHERES, 0)
    r.publish(1, 1)
    r.take()
    two = r.install(SPHERES, 0)
    r.publish(1, 2)
    three = r.install(SPHERES, 0)
    assert r.retired() == [two], "never read, so free at once"
    assert {one, three} <= set(r.live()), "the front's and the current one are still live"
    r.close()


@pytest.mark.gpu
def test_gpu_frames_carry_the_steps_pictures():
    """A sphere world steps and keeps every step in the ring; the reader takes now and then and finds, in the slot
    it is handed, exactly the picture the world showed at that step."""
    import sphere_cases as SC
    from vxr import spheres as S
    s = SC.until_done_pile()
    s.start("gpu")
    r = ShownRing()
    r.install(SPHERES, s.n, (s.sx, s.sy, s.sz))
    seen = {}
    for step in range(1, 13):
        s.advance(1)
        seen[step] = s.shown().copy()
        r.keep(s.world, step)
        if step % 4 == 0:
            f = r.take()
            assert f.step == step and f.words == s.n * S.SHOWN_STRIDE
            assert np.array_equal(ShownRing.read(f), seen[step])
    r.close()
    s.close()
