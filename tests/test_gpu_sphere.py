"""The sphere package on the GPU, through the C-ABI: the reference's sphere tests (sphere_cases.py) with their own
tolerances, and every snapshot equal to the oracle's bit for bit (the kernels keep the reference's arithmetic in
its association order; the list, the sort and every sum are in the oracle's order)."""
import numpy as np
import pytest

import sphere_cases as C
from sphere_scene import SphereScene
from vxr import spheres as S

pytestmark = pytest.mark.gpu


def same(a_snaps, b_snaps):
    assert len(a_snaps) == len(b_snaps)
    for k, (a, b) in enumerate(zip(a_snaps, b_snaps)):
        for name in a:
            x, y = a[name], b[name]
            if not np.array_equal(x.view(np.int32), y.view(np.int32)):
                bad = np.flatnonzero(x.view(np.int32) != y.view(np.int32))
                raise AssertionError(f"snapshot {k}, {name}: {len(bad)} words differ, first at {bad[0]}: "
                                     f"{x[bad[0]]!r} against {y[bad[0]]!r}")


def both(case, *args):
    gpu = case("gpu", *args)
    oracle = case("oracle", *args)
    same(gpu, oracle)


@pytest.mark.parametrize("solve", C.EVERY_SOLVE, ids=["jacobi", "gauss_seidel"])
@pytest.mark.parametrize("case", C.EVERY_SOLVE_CASES, ids=lambda c: c.__name__)
def test_gpu_every_solve(case, solve):
    both(case, solve)


@pytest.mark.parametrize("case", C.FRICTION_CASES, ids=lambda c: c.__name__)
def test_gpu_friction(case):
    both(case)


def test_gpu_grid_finds_every_pair():
    both(C.case_grid_finds_every_pair)


@pytest.mark.parametrize("grid,solve,mu", [(False, S.JACOBI, 0.0), (True, S.JACOBI, 0.0),
                                           (True, S.GAUSS_SEIDEL_BY_CONTACT, 0.0),
                                           (True, S.GAUSS_SEIDEL_BY_CONTACT, 0.5)],
                         ids=["pairs-jacobi", "grid-jacobi", "gauss-seidel", "gauss-seidel-friction"])
def test_gpu_dropped_pile(grid, solve, mu):
    both(C.case_dropped_pile, grid, solve, mu)


def test_gpu_friction_pile_rests():
    both(C.case_friction_pile_rests)


def test_gpu_until_done_is_enough_fixed_rounds():
    both(C.case_until_done)


def run_scene(make, backend, steps, **kw):
    scene = make()
    scene.start(backend, **kw)
    reports = [scene.world.step() for _ in range(steps)]
    out = C.snapshot(scene)
    ab, done, imp = scene.world.contact_list()
    return scene, reports, out, (ab, done, imp), scene.world.walls(), scene.world.counts()


def compare_runs(make, steps, gpu_kw=None):
    g = run_scene(make, "gpu", steps, **(gpu_kw or {}))
    o = run_scene(make, "oracle", steps)
    try:
        assert g[1] == o[1], "the reports (waits, rounds, most rounds, unlisted) differ"
        same([g[2]], [o[2]])
        for a, b in zip(g[3], o[3]):
            assert np.array_equal(a.view(np.int32), b.view(np.int32)), "the contact lists differ"
        assert np.array_equal(g[4].view(np.int32), o[4].view(np.int32)), "the wall impulses differ"
        assert np.array_equal(g[5], o[5]), "the list's counts differ"
    finally:
        g[0].close()
        o[0].close()
    return g


def test_gpu_list_reports_and_walls_match_the_oracle():
    """Ten steps of the crowded until-done pile with friction: the list in list order with its done marks and
    impulses, the wall impulses, the counts and every step's report equal the oracle's."""
    def make():
        s = C.until_done_pile()
        s.mu_static = s.mu_kinetic = 0.5
        s.mu_rolling = 0.05
        s.restitution = 0.3
        return s
    compare_runs(make, 10)


@pytest.mark.parametrize("blocks", [2, 7])
def test_gpu_many_blocks_match_the_oracle(blocks):
    """The same scene on a cooperative grid of several blocks (the grid barrier between passes)."""
    def make():
        s = C.until_done_pile()
        s.mu_static = s.mu_kinetic = 0.5
        s.restitution = 0.2
        return s
    g = compare_runs(make, 6, gpu_kw={"blocks": blocks})
    assert g[0] is not None


@pytest.mark.parametrize("cluster", [4, 8, 16])
def test_gpu_a_cluster_matches_the_oracle(cluster):
    """The step on one thread-block cluster (the cluster's barrier between passes): the same as the oracle."""
    def make():
        s = C.until_done_pile()
        s.mu_static = s.mu_kinetic = 0.5
        s.mu_rolling = 0.05
        s.restitution = 0.2
        return s
    compare_runs(make, 8, gpu_kw={"cluster": cluster})


def test_gpu_a_cluster_runs_the_lattice_as_the_oracle_does():
    compare_runs(lattice_scene, 90, gpu_kw={"cluster": 8})


def test_gpu_an_overfull_list_counts_what_did_not_fit():
    """With one list place a sphere, a crowded pile leaves contacts unlisted; the GPU counts and drops the same
    ones as the oracle."""
    def make():
        s = C.until_done_pile()
        return s
    g = run_scene(make, "gpu", 3, contacts_per_sphere=1)
    o = run_scene(make, "oracle", 3, per_sphere=1)
    try:
        assert g[1] == o[1]
        assert sum(r[3] for r in g[1]) > 0, "the scene overfills a list of one place a sphere"
        same([g[2]], [o[2]])
        assert np.array_equal(g[5], o[5])
    finally:
        g[0].close()
        o[0].close()


def lattice_scene(steps_seed=1):
    from vxr import scenes
    sc = scenes.sphere_lattice(seed=steps_seed)
    scene = SphereScene(sc["spheres"])
    for k in ("x", "y", "z", "r", "im"):
        getattr(scene, k)[:] = sc[k]
    scene.sx, scene.sy, scene.sz = sc["walls"]
    scene.dt, scene.substeps, scene.iterations = sc["dt"], sc["substeps"], sc["iterations"]
    scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
    scene.restitution = 0.2
    scene.mu_static = scene.mu_kinetic = 0.5
    return scene


def test_gpu_sphere_lattice_matches_the_oracle():
    """The plain sphere scene (1,024 spheres, 4 substeps, 8 iterations, mu 0.5, e 0.2): 90 steps (the lattice lands
    and piles) equal to the oracle bit for bit, reports included."""
    compare_runs(lattice_scene, 90)


def test_gpu_start_matches_the_reference_start():
    """SphereSimulation.start: the picture's before and after are the start state; the state reads back."""
    from vxr.sphere_simulation import SphereSimulation
    sc = lattice_scene()
    with SphereSimulation(sc.n, 4, 8, S.covering(sc.sx, sc.sy, sc.sz, 1.0), S.GAUSS_SEIDEL_BY_CONTACT) as sim:
        sim.start(sc.x, sc.y, sc.z, sc.u, sc.v, sc.w, sc.r, sc.im, sc.param_bits())
        shown = sim.read_shown().reshape(sc.n, S.SHOWN_STRIDE)
        assert np.array_equal(shown[:, 0], sc.x) and np.array_equal(shown[:, 4], sc.x)
        assert np.all(shown[:, S.TURNED_AFTER + 3] == 1)
        x, y, z, u, v, w, ax, ay, az = sim.state()
        assert np.array_equal(y, sc.y) and np.all(u == 0)
        sim.step_and_wait()
        later = sim.read_shown().reshape(sc.n, S.SHOWN_STRIDE)
        assert np.array_equal(later[:, 1], sc.y), "the step before's centre moved to the before slot"
        assert sim.launches() == 1


def test_gpu_steps_in_one_call_equal_steps_one_by_one():
    """A call of many steps (one launch) leaves what as many calls of one step leave."""
    from vxr.sphere_simulation import SphereSimulation
    sc = C.until_done_pile()
    sc.mu_static = sc.mu_kinetic = 0.5
    grid = S.covering(sc.sx, sc.sy, sc.sz, sc.widest())
    fields = {"x": sc.x, "y": sc.y, "z": sc.z, "r": sc.r, "im": sc.im}
    outs = []
    for per_call in (1, 5):
        with SphereSimulation(sc.n, sc.substeps, 1, grid, S.GAUSS_SEIDEL_BY_CONTACT) as sim:
            sim.load_state(fields, sc.param_bits())
            for _ in range(10 // per_call):
                sim.step_and_wait(per_call)
            outs.append([sim.field(k) for k in S.FIELDS] + [sim.read_shown()])
            assert sim.launches() == 10 // per_call
    for a, b in zip(*outs):
        assert np.array_equal(a.view(np.int32), b.view(np.int32))


def test_gpu_bad_config_is_refused():
    from vxr._lib import VxrError
    from vxr.sphere_simulation import SphereSimulation, make_params
    with pytest.raises(VxrError):
        SphereSimulation(10, 1, 1, None, S.GAUSS_SEIDEL_BY_CONTACT)  # Gauss-Seidel needs the grid
    with pytest.raises(VxrError):
        SphereSimulation(S.MOST_LISTED_SPHERES + 1, 1, 1, S.SphereGrid(4, 4, 4, 1.0), S.GAUSS_SEIDEL_BY_CONTACT)
    with pytest.raises(VxrError):
        make_params(0.01, 0, -9.81, 0, 1, 1, 1, 2.0, True)
    assert np.array_equal(make_params(0.01, 0, -9.81, 0, 1, 1, 1, 1, True, 0.2, 0.5, 0.5, 0.1),
                          S.params(0.01, 0, -9.81, 0, 1, 1, 1, 1, True, 0.2, 0.5, 0.5, 0.1))


@pytest.mark.parametrize("solver", ["until done mu=0.5", "until done", "grid averaged omega=1"])
def test_gpu_the_reference_pile_matches_the_oracle(solver):
    """The reference's own sphere benchmark scene (its sweep's large pile, 4,096 spheres) with each of the solver
    settings it publishes times for: 60 frames, through the drop onto the floor, every field equal to the oracle's."""
    from oracle.sphere import OracleSphereWorld
    from vxr import scenes
    from vxr.sphere_simulation import SphereSimulation
    sc = scenes.sphere_pile(solver=solver)
    n = sc["spheres"]
    g = SphereSimulation(n, sc["substeps"], sc["iterations"], sc["grid"], sc["solve"])
    g.start(sc["x"], sc["y"], sc["z"], sc["u"], sc["v"], sc["w"], sc["r"], sc["im"], sc["params"])
    g.friction(sc["friction"])
    o = OracleSphereWorld(n, sc["substeps"], sc["iterations"], sc["solve"], sc["grid"])
    for k in ("x", "y", "z", "u", "v", "w", "r", "im"):
        o.set_field(k, sc[k])
    o.set_shown(S.shown_at_start(sc["x"], sc["y"], sc["z"], sc["r"]))
    o.set_params(sc["params"], sc["friction"])
    g.step_and_wait(60)
    o.step(60)
    for name in S.FIELDS:
        assert np.array_equal(g.field(name).view(np.int32), o.field(name).view(np.int32)), name
    assert np.array_equal(g.read_shown().view(np.int32), o.shown().view(np.int32))
    g.close()
    o.close()
