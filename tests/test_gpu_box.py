"""The CUDA box/mixed step against the oracle and the reference's known-answer tests, through the C-ABI.

Parity bar: the broad phase's candidate pair set bit-exact (sorted); manifolds, states and impulses equal to the
oracle's as f32 values (the kernels keep the reference's association order, compiled without contraction, so the
stated tolerances 1e-5 relative on positions and 1e-4 on impulses are met with room to spare — equality is
asserted, and a tolerance-based check reports the largest difference when it fails).
"""
import numpy as np
import pytest

import box_cases as C
from box_scene import BoxScene
from test_oracle_contact import CASES, check_random_pairs, collide_backend, random_pairs
from vxr import boxes as B

pytestmark = pytest.mark.gpu

POS_REL = 1e-5
IMPULSE_ABS = 1e-4


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.__name__)
def test_gpu_hand_cases(case):
    case("gpu")


def manifold_words(m):
    """The words of a manifold the step reads: normal, count, axis and the count points."""
    cnt = int(m[B.COUNT])
    return np.concatenate([m[:5], m[8:8 + 8 * cnt]])


def test_gpu_random_pairs_match_the_oracle():
    solids = random_pairs()
    gpu = collide_backend("gpu", 0, *solids)
    check_random_pairs(solids, gpu)
    orc = collide_backend("oracle", 0, *solids)
    for p in range(len(solids) // 2):
        g, o = gpu[40 * p:40 * p + 40], orc[40 * p:40 * p + 40]
        assert g[B.COUNT] == o[B.COUNT], p
        if o[B.COUNT] > 0:
            np.testing.assert_array_equal(manifold_words(g), manifold_words(o), err_msg=f"pair {p}")


def run_both(make_scene, steps, **kw):
    a = make_scene()
    b = make_scene()
    a.start("oracle", threads=True)
    b.start("gpu", **kw)
    ra = rb = None
    for _ in range(steps):
        ra = a.world.step(1)
        rb = b.world.step(1)
        assert tuple(ra) == tuple(rb), (tuple(ra), tuple(rb))
    return a, b


def compare_worlds(a, b, exact=True):
    a.read()
    b.read()
    fa = [a.x, a.y, a.z, a.u, a.v, a.w, a.l[0], a.l[1], a.l[2], a.q[0], a.q[1], a.q[2], a.q[3]]
    fb = [b.x, b.y, b.z, b.u, b.v, b.w, b.l[0], b.l[1], b.l[2], b.q[0], b.q[1], b.q[2], b.q[3]]
    names = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]
    for name, va, vb in zip(names, fa, fb):
        if name in ("x", "y", "z"):
            np.testing.assert_allclose(vb, va, rtol=POS_REL, atol=0, err_msg=name)
        if exact:
            np.testing.assert_array_equal(vb, va, err_msg=name)
    pa = a.world.touching_pairs()
    pb = b.world.touching_pairs()
    assert pa == pb
    ma = np.array(a.world.touching_manifolds()).reshape(-1, 40)
    mb = np.array(b.world.touching_manifolds()).reshape(-1, 40)
    for k in range(len(pa)):
        np.testing.assert_array_equal(manifold_words(mb[k]), manifold_words(ma[k]), err_msg=f"manifold {k}")
    ia = np.array(a.world.touching_impulses()).reshape(-1, 28)
    ib = np.array(b.world.touching_impulses()).reshape(-1, 28)
    np.testing.assert_allclose(ib, ia, atol=IMPULSE_ABS, rtol=0)
    if exact:
        np.testing.assert_array_equal(ib, ia)


def test_gpu_broad_phase_is_the_oracles_pair_set():
    scene_o = C.broad_fixture()
    scene_g = C.broad_fixture()
    scene_o.start("oracle")
    scene_g.start("gpu")
    scene_o.advance(1)
    scene_g.advance(1)
    co = scene_o.world.candidate_pairs()
    cg = scene_g.world.candidate_pairs()
    np.testing.assert_array_equal(cg, co)
    assert scene_o.world.touching_pairs() == scene_g.world.touching_pairs()


def test_gpu_grid_finds_every_pair():
    C.case_grid_finds_every_pair("gpu")


def test_gpu_single_step_of_a_pile_matches_the_oracle():
    a, b = run_both(lambda: C.pile_scene(7), 1)
    compare_worlds(a, b)


def test_gpu_pile_steps_match_the_oracle_bit_for_bit():
    a, b = run_both(lambda: C.pile_scene(7), 40)
    compare_worlds(a, b)
    la, ra, oa = a.world.buffer("lambda"), a.world.buffer("rub"), a.world.buffer("roll")
    lb, rb, ob = b.world.walls()
    np.testing.assert_array_equal(lb, la)
    np.testing.assert_array_equal(rb, ra)


def test_gpu_mixed_pile_steps_match_the_oracle_bit_for_bit():
    a, b = run_both(C.mixed_pile_scene, 40)
    compare_worlds(a, b)
    lb, rb, ob = b.world.walls()
    np.testing.assert_array_equal(ob, a.world.buffer("roll"))


@pytest.mark.parametrize("schedule", [0, 1], ids=["barrier", "dependency"])
def test_gpu_symmetric_sweeps_match_the_oracle(schedule):
    def make():
        s = C.mixed_pile_scene()
        s.symmetric = True
        s.passes = 3
        return s
    a, b = run_both(make, 20, schedule=schedule)
    compare_worlds(a, b)


def test_gpu_dependency_schedule_matches_the_oracle():
    a, b = run_both(lambda: C.pile_scene(7), 30, schedule=1)
    compare_worlds(a, b)


def test_gpu_fixed_bodies_and_spheres_match_the_oracle():
    """A mixed pile on four fixed balls and a fixed slab: fixed bodies take part in pairs (their angular
    momentum is written, as the reference writes it) and stiffen their contacts."""
    def make():
        s = C.mixed_pile_scene()
        for k in range(0, 8):
            s.im[k] = 0.0
        return s
    a, b = run_both(make, 30)
    compare_worlds(a, b)


def test_gpu_show_matches_the_oracle():
    a, b = run_both(lambda: C.column_scene(10), 3)
    np.testing.assert_array_equal(b.world.shown(), a.world.shown())


KNOWN = [C.case_free_fall, C.case_stable_spin, C.case_tumble_keeps_momentum_and_energy, C.case_head_on,
         C.case_column, C.case_flat_rests_flat, C.case_slope_holds, C.case_slope_slides, C.case_ball_rests_on_box,
         C.case_sliding_ball_rolls, C.case_rolling_resistance, C.case_ball_into_box, C.case_show,
         C.case_mixed_pile_rests]


@pytest.mark.parametrize("case", KNOWN, ids=lambda c: c.__name__)
def test_gpu_known_answer(case):
    case("gpu")


def test_gpu_pile_of_343_rests():
    C.case_pile("gpu")


def test_gpu_pile_of_1000_rests():
    C.case_pile("gpu", side=10, most_energy=1e-5, most_depth=2e-3)


def test_gpu_measuring_the_residual_changes_nothing():
    a = C.pile_scene(7)
    b = C.pile_scene(7)
    a.start("oracle", threads=True)
    b.start("gpu")
    b.world.measure(residual=True)
    for _ in range(30):
        assert tuple(a.world.step(1)) == tuple(b.world.step(1))
    compare_worlds(a, b)
    res, used = b.world.residuals()
    assert res.shape == (b.substeps, 2 * b.passes + 1)
    assert (res[:, 0] == 0).all()  # the warm sweep moves no impulse
    assert (used == b.passes).all()
    pairs, walls = b.world.residual_parts()  # the pile's pairs and its floor contacts, each part apart
    assert np.array_equal(np.maximum(pairs, walls), res)
    assert (pairs[:, 1:] > 0).any() and (walls[:, 1:] > 0).any()


def test_gpu_first_substeps_alone_and_solve_only():
    """The measurement switch: a step of only the first substep, its relax sweeps skipped, runs that substep's
    solve sweeps and nothing after them; whole steps afterwards run every substep's solve and relax sweeps."""
    scene = C.pile_scene(7)
    scene.start("gpu")
    w = scene.world
    w.step(5)
    w.measure(residual=True)
    w.first_substeps(1, solve_only=True)
    w.step(1)
    res, used = w.residuals()
    assert used[0, 0] == scene.passes and used[0, 1] == 0
    assert (res[0, 1:1 + scene.passes] > 0).any() and (res[0, 1 + scene.passes:] == 0).all()
    assert (res[1:] == 0).all()
    w.first_substeps(0)
    w.step(1)
    res, used = w.residuals()
    assert (used == scene.passes).all()
    with pytest.raises(Exception):
        w.first_substeps(scene.substeps + 1)
    scene.close()


def iterations(world, steps, cold, tolerance=1e-4, cap=64):
    world.measure(residual=True, cold_start=cold, sweeps=cap, tolerance=tolerance)
    runs = []
    for _ in range(steps):
        world.step(1)
        res, used = world.residuals()
        for sub in range(used.shape[0]):
            n = used[sub, 0]
            assert n <= cap
            if n < cap:  # it stopped: that sweep's residual met the tolerance
                assert res[sub, n] <= tolerance
            runs.append(n)
    return float(np.mean(runs))


def test_gpu_a_warm_start_converges_in_fewer_sweeps_than_a_cold_one():
    scene = C.pile_scene(7)
    scene.passes = 64
    scene.start("gpu")
    scene.world.measure(residual=True, sweeps=8)
    scene.advance_seconds(3)  # the pile at rest
    warm = iterations(scene.world, 5, cold=False)
    cold = iterations(scene.world, 5, cold=True)
    assert warm < cold, (warm, cold)


def test_gpu_towers_match_the_oracle():
    """The box-stacking configuration's towers, a 2 x 2 block 16 high, at its 8 substeps and 16 sweeps: after
    every 20 of 100 steps every state word equals the oracle's, to the bit (the towers settle, lean and start to
    topple over these steps)."""
    from oracle.box import OracleBoxWorld
    from vxr import scenes
    from vxr.box_simulation import BoxSimulation
    sc = scenes.towers(seed=5, towers_x=2, towers_z=2, height=16)
    o = OracleBoxWorld(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"], threads=True)
    for k in scenes.FIELDS:
        o.set_field(k, sc[k])
    o.set_params(sc["params"])
    g = BoxSimulation(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"])
    g.load_state([sc[k] for k in scenes.FIELDS], sc["params"])
    names = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]
    for _ in range(5):
        o.step(20)
        g.step_and_wait(20)
        got = g.state()
        for name, a in zip(names, got):
            assert np.array_equal(a.view(np.int32), o.field(name).view(np.int32)), name
    assert g.touching_pairs() == o.touching_pairs()
    o.close()
    g.close()


@pytest.mark.parametrize("tiled", [False, True], ids=["per-thread", "tiled"])
@pytest.mark.parametrize("bodies", [8000, 16000], ids=["staged", "global"])
def test_gpu_crowded_broad_phase_keeps_the_first_32_found(bodies, tiled):
    """Small spheres crowded into one cubic metre, dozens of partners a body: each body's slots hold the first 32
    bodies the reference's walk finds, sorted (BoxBroad.list :103-164), and the rest are counted unlisted. 8,000
    bodies keep every block's neighbourhood within its shared memory; 16,000 overflow it, so the tiled list reads
    those neighbourhoods from global memory. Candidate pairs, the report and the step's state equal the oracle's."""
    from oracle.box import OracleBoxWorld
    from vxr.box_simulation import BoxSimulation
    rng = np.random.Generator(np.random.PCG64(12))
    r = 0.05
    f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    x, y, z = (f32(rng.uniform(1.5, 2.5, bodies)) for _ in range(3))
    zero = np.zeros(bodies, np.float32)
    fields = {"x": x, "y": y, "z": z, "u": zero, "v": zero, "w": zero, "lx": zero, "ly": zero, "lz": zero,
              "qx": zero, "qy": zero, "qz": zero, "qw": np.ones(bodies, np.float32),
              "im": np.full(bodies, 1.0 / 0.5, np.float32), "hx": np.full(bodies, r, np.float32),
              "hy": np.full(bodies, r, np.float32), "hz": np.full(bodies, r, np.float32),
              "shape": np.full(bodies, B.SPHERE_SHAPE, np.float32)}
    order = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw", "im", "hx", "hy", "hz", "shape"]
    grid = B.grid(4.0, 4.0, 4.0, r, 0.005)
    params = B.params(1 / 240, 0.0, -9.81, 0.0, 4.0, 4.0, 4.0, 0.5, 0.5, 0.005, 0.1)
    o = OracleBoxWorld(bodies, 1, 2, False, grid, threads=True)
    for k in order:
        o.set_field(k, fields[k])
    o.set_params(params)
    g = BoxSimulation(bodies, 1, 2, False, grid)
    g.load_state([fields[k] for k in order], params)
    g.list_kernel(tiled)
    ro = o.step(1)
    rg = g.step_and_wait(1)
    assert ro == tuple(rg)
    assert ro[4] > 0  # bodies with more than 32 partners
    np.testing.assert_array_equal(g.candidate_pairs(), o.candidate_pairs())
    for name, a in zip(order[:13], g.state()):
        assert np.array_equal(a.view(np.int32), o.field(name).view(np.int32)), name
    o.close()
    g.close()


def test_gpu_tiled_list_matches_the_per_thread_walk_through_the_drop():
    """The two list kernels on 16,384 bodies of the large mixed scene through 120 steps of its drop (sparse air,
    a crowding floor): the same candidate pairs every 20 steps and the same state."""
    from vxr import scenes
    from vxr.box_simulation import BoxSimulation
    sc = scenes.sub_volume(262_144, 16_384 / 262_144, seed=13)
    worlds = []
    for tiled in (False, True):
        w = BoxSimulation(sc["bodies"], sc["substeps"], sc["sweeps"], False, sc["grid"])
        w.load_state([sc[k] for k in scenes.FIELDS], sc["params"])
        w.list_kernel(tiled)
        worlds.append(w)
    for _ in range(6):
        ra = worlds[0].step_and_wait(20)
        rb = worlds[1].step_and_wait(20)
        assert tuple(ra) == tuple(rb)
        np.testing.assert_array_equal(worlds[1].candidate_pairs(), worlds[0].candidate_pairs())
        for x, y in zip(worlds[1].state(), worlds[0].state()):
            assert np.array_equal(x.view(np.int32), y.view(np.int32))
    for w in worlds:
        w.close()


def test_gpu_state_read_back_without_waiting_equals_the_waited_one():
    """Steps read back with vxr_box_state_async into two sets of arrays in turn (each copy travelling while the next
    step runs) give, step by step, the very words a twin world's waited read-back gives."""
    a = C.mixed_pile_scene()
    b = C.mixed_pile_scene()
    a.start("gpu")
    b.start("gpu")
    n = a.n
    sets = [[np.zeros(n, np.float32) for _ in range(13)] for _ in range(2)]
    want = []
    for k in range(6):
        a.world.step_async(1)
        a.world.state_async(sets[k % 2], k % 2)
        b.world.step(1)
        want.append([x.copy() for x in b.world.state()])
        if k > 0:
            a.world.state_wait((k - 1) % 2)
            for x, y in zip(sets[(k - 1) % 2], want[k - 1]):
                assert np.array_equal(x.view(np.int32), y.view(np.int32)), f"step {k}"
    a.world.state_wait(1)
    for x, y in zip(sets[1], want[5]):
        assert np.array_equal(x.view(np.int32), y.view(np.int32))
    a.world.sync()
    a.close()
    b.close()
