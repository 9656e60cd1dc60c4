"""Batched scenes on the GPU (vxr_box_create_batch): every scene of a batch steps as a world of that scene alone
would, bit for bit against the oracle run scene by scene; and steps replayed from a captured CUDA graph equal the
same steps enqueued one by one."""
import numpy as np
import pytest

from vxr import scenes
from vxr.box_simulation import BatchSimulation, BoxSimulation

pytestmark = pytest.mark.gpu

STATE = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]


def small_batch(seed=3, count=5, largest=300):
    return scenes.batched(scenes=count, seed=seed, smallest=40, largest=largest)


def gpu_batch(b, steps, graph=False, **kw):
    sim = BatchSimulation(b["counts"], b["grids"], b["substeps"], b["sweeps"], **kw)
    sim.load_state([b[k] for k in scenes.FIELDS], None)
    sim.scene_params(b["params"])
    if graph:
        assert steps % 2 == 0
        sim.step_graph(steps // 2)
        sim.sync()
    else:
        sim.step_and_wait(steps)
    out = dict(zip(STATE, sim.state()))
    shown = sim.read_shown()
    first = sim.first.copy()
    launches = sim.launches()
    sim.close()
    return out, shown, first, launches


def oracle_scene(part, params, steps):
    from oracle.box import OracleBoxWorld
    w = OracleBoxWorld(part["bodies"], part["substeps"], part["sweeps"], False, part["grid"])
    for k in scenes.FIELDS:
        w.set_field(k, part[k])
    w.set_params(params)
    w.step(steps)
    out = {k: w.field(k) for k in STATE}
    w.close()
    return out


def test_gpu_batch_scenes_each_match_the_oracle():
    """Five scenes of 40-300 bodies, each with its own gravity tilt, friction and walls, 60 steps (they land and
    pile): each scene's bodies equal the oracle's run of that scene alone, to the bit."""
    b = small_batch()
    steps = 60
    out, _, first, _ = gpu_batch(b, steps)
    for sc, part in enumerate(b["parts"]):
        want = oracle_scene(part, b["params"][sc], steps)
        lo, hi = first[sc], first[sc + 1]
        for k in STATE:
            got = out[k][lo:hi]
            assert np.array_equal(got.view(np.int32), want[k].view(np.int32)), f"scene {sc}, {k}"


@pytest.mark.parametrize("schedule", [0, 1], ids=["barrier", "dependency"])
def test_gpu_graph_replays_equal_plain_steps(schedule):
    """20 steps as 10 replays of a captured pair of steps leave what 20 enqueued steps leave (state and picture),
    and the launch count is the kernels of the graph times its replays."""
    b = small_batch(seed=5, count=4, largest=500)
    plain, shown_p, _, launches_p = gpu_batch(b, 20, schedule=schedule)
    graph, shown_g, _, launches_g = gpu_batch(b, 20, graph=True, schedule=schedule)
    for k in STATE:
        assert np.array_equal(plain[k].view(np.int32), graph[k].view(np.int32)), k
    assert np.array_equal(shown_p.view(np.int32), shown_g.view(np.int32))
    assert launches_g == launches_p


def test_gpu_graph_on_a_single_scene_world():
    """A plain world steps through a captured graph too, and changing the parameters captures it again."""
    sc = scenes.large_mixed(4096, seed=2, volume=(24.0, 12.0, 24.0))
    def make():
        w = BoxSimulation(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"])
        l = [sc["lx"], sc["ly"], sc["lz"]]
        q = [sc["qx"], sc["qy"], sc["qz"], sc["qw"]]
        h = [sc["hx"], sc["hy"], sc["hz"]]
        w.start_momentum(sc["x"], sc["y"], sc["z"], sc["u"], sc["v"], sc["w"], l, q, h, sc["shape"], sc["im"],
                         sc["params"])
        return w
    a, g = make(), make()
    a.step_and_wait(8)
    g.step_graph(2)
    g.sync()
    g.params(sc["params"])  # new parameters: the next call captures again
    g.step_graph(2)
    g.sync()
    for x, y in zip(a.state(), g.state()):
        assert np.array_equal(x.view(np.int32), y.view(np.int32))
    a.close()
    g.close()


def test_gpu_batch_refuses_mismatched_shared_words():
    from vxr._lib import VxrError
    b = small_batch(count=2, largest=80)
    sim = BatchSimulation(b["counts"], b["grids"], b["substeps"], b["sweeps"])
    bad = b["params"].copy()
    bad[1, 0] = np.array([1 / 500], np.float32).view(np.int32)[0]  # another substep length
    with pytest.raises(VxrError):
        sim.scene_params(bad)
    sim.load_state([b[k] for k in scenes.FIELDS], None)
    with pytest.raises(VxrError):
        sim.step_and_wait(1)  # no scene parameters yet
    sim.close()
