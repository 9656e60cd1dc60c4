"""Pins the sphere oracle (oracle/sphere_oracle.cpp) to the reference's own sphere tests, restated in
sphere_cases.py with the reference's tolerances, plus the host helpers of vxr/spheres.py."""
import numpy as np
import pytest

import sphere_cases as C
from vxr import spheres as S


@pytest.mark.parametrize("solve", C.EVERY_SOLVE, ids=["jacobi", "gauss_seidel"])
@pytest.mark.parametrize("case", C.EVERY_SOLVE_CASES, ids=lambda c: c.__name__)
def test_oracle_every_solve(case, solve):
    case("oracle", solve)


@pytest.mark.parametrize("case", C.FRICTION_CASES, ids=lambda c: c.__name__)
def test_oracle_friction(case):
    case("oracle")


def test_oracle_grid_finds_every_pair():
    C.case_grid_finds_every_pair("oracle")


@pytest.mark.parametrize("grid,solve,mu", [(False, S.JACOBI, 0.0), (True, S.JACOBI, 0.0),
                                           (True, S.GAUSS_SEIDEL_BY_CONTACT, 0.0),
                                           (True, S.GAUSS_SEIDEL_BY_CONTACT, 0.5)],
                         ids=["pairs-jacobi", "grid-jacobi", "gauss-seidel", "gauss-seidel-friction"])
def test_oracle_dropped_pile(grid, solve, mu):
    C.case_dropped_pile("oracle", grid, solve, mu)


def test_oracle_friction_pile_rests():
    C.case_friction_pile_rests("oracle")


def test_oracle_until_done_is_enough_fixed_rounds():
    C.case_until_done("oracle")


def test_grid_covers_the_box():
    """GridTest.aGridCoversTheBoxWithCellsAsWideAsTheWidestSphere."""
    grid = S.covering(1, 0.45, 0.1, 0.1)
    assert (grid.nx, grid.ny, grid.nz, grid.cells()) == (10, 5, 1, 50)
    with pytest.raises(ValueError):
        S.covering(1, 1, 1, 0)


def test_params_are_checked_and_rubs_read_from_them():
    """Spheres.params throws on bad values; Spheres.rubs reads friction from the words."""
    with pytest.raises(ValueError):
        S.params(0, 0, -9.81, 0, 1, 1, 1, 1, True)
    with pytest.raises(ValueError):
        S.params(0.01, 0, -9.81, 0, 1, 1, 1, 1.5, True)
    with pytest.raises(ValueError):
        S.params(0.01, 0, -9.81, 0, 1, 1, 1, 1, True, restitution=1.5)
    with pytest.raises(ValueError):
        S.params(0.01, 0, -9.81, 0, 1, 1, 1, 1, True, mu_static=-1)
    words = S.params(0.01, 0, -9.81, 0, 1, 1, 1, 1, True)
    assert not S.rubs(words)
    assert words.view(np.float32)[S.AVERAGED] == 1
    assert S.rubs(S.params(0.01, 0, -9.81, 0, 1, 1, 1, 1, True, mu_rolling=0.1))


def test_oracle_list_is_every_near_pair_once():
    """listContacts: every pair within 1.02 (ra + rb), once, lower index first; impulses carried by partner."""
    scene = C.until_done_pile()
    with scene:
        scene.start("oracle").advance(3)
        ab, done, imp = scene.world.contact_list()
        x = np.stack([scene.floats("x"), scene.floats("y"), scene.floats("z")], 1).astype(np.float64)
        assert len(ab) > 0 and np.all(ab[:, 0] < ab[:, 1])
        assert len({(int(a), int(b)) for a, b in ab}) == len(ab)
        # every pair listed was near at the list's time; nothing far is listed (positions have since moved a little)
        r = scene.r.astype(np.float64)
        d = np.linalg.norm(x[ab[:, 0]] - x[ab[:, 1]], axis=1)
        assert np.all(d < 1.2 * (r[ab[:, 0]] + r[ab[:, 1]]))
        assert np.all(done == 1)  # the last pass of the last substep solved every contact
