"""Known-answer cases of the reference's sphere tests, each a function of the backend (and the solve).

Restated from vexelray-sim-rigid-core/src/test/java/dev/vexelray/sim/rigid/sphere/: SpheresTest.java,
BounceTest.java, FrictionTest.java, RollingTest.java, SpinTest.java, PressingTest.java, PileTest.java, GridTest.java
and UntilDoneTest.java, with the reference's tolerances. Each case asserts the reference's physics and returns the
snapshots it took, so that test_gpu_sphere.py can also hold the CUDA library to the oracle bit for bit.
test_oracle_sphere.py runs them on the oracle (pinning it).
"""
import math

import numpy as np

from java_random import JavaRandom
from sphere_scene import SphereScene
from vxr import spheres as S

G = 9.81
f32 = np.float32

EVERY_SOLVE = [S.JACOBI, S.GAUSS_SEIDEL_BY_CONTACT]


def snapshot(scene):
    """Every per-sphere field and the picture's buffer, as the backend holds them now."""
    out = {name: scene.floats(name).copy() for name in S.FIELDS}
    out["shown"] = scene.shown().copy()
    return out


# --- SpheresTest (:39-115) ------------------------------------------------------------------------------------------

def case_fall(backend, solve):
    """aFallingSphereFollowsSymplecticEulerExactly: v = -g h k and y = y0 - g h^2 k (k + 1) / 2 after k substeps."""
    with SphereScene(1).uniform(0.1, 1) as scene:
        scene.sx = scene.sy = scene.sz = 10
        scene.x[0] = scene.z[0] = 5
        scene.y[0] = 8
        scene.solve = solve
        scene.start(backend).advance(30)
        scene.read()
        k = 30 * scene.substeps
        h = scene.dt / scene.substeps
        assert abs(-9.81 * h * k - scene.v[0]) <= 1e-4, "velocity"
        assert abs(8 - 9.81 * h * h * k * (k + 1) / 2 - scene.y[0]) <= 1e-4, "height"
        assert scene.x[0] == 5, "nothing moves it sideways"
        return [snapshot(scene)]


def case_rest_on_floor(backend, solve):
    """aDroppedSphereComesToRestOnTheFloor."""
    with SphereScene(1).uniform(0.1, 1) as scene:
        scene.x[0] = scene.z[0] = 0.5
        scene.y[0] = 0.8
        scene.solve = solve
        scene.start(backend).advance_seconds(1)
        state = scene.diagnostics()
        assert abs(0.1 - scene.y[0]) <= 1e-6, "resting on the floor"
        assert state.max_speed < 1e-4, f"at rest: {state}"
        assert state.max_wall < 1e-5, f"not in the floor: {state}"
        return [snapshot(scene)]


def case_inelastic_collision(backend, solve):
    """aCollisionKeepsMomentumAndTheSpheresLeaveTogether: 1 kg at 2 m/s into 3 kg, both leave at 0.5 m/s."""
    with SphereScene(2).uniform(0.1, 1) as scene:
        scene.gy = 0
        scene.sx = 4
        scene.y[:] = 0.5
        scene.z[:] = 0.5
        scene.x[0] = 1
        scene.x[1] = 2
        scene.u[0] = 2
        scene.im[1] = f32(1 / 3)
        scene.solve = solve
        scene.start(backend).advance_seconds(1)
        state = scene.diagnostics()
        assert abs(2 - state.momentum[0]) <= 1e-6, f"momentum: {state}"
        assert abs(0.5 - scene.u[0]) <= 1e-3, "the light one"
        assert abs(0.5 - scene.u[1]) <= 1e-3, "the heavy one"
        assert scene.x[0] < scene.x[1], "they did not pass through each other"
        assert state.max_overlap < 1e-3, f"touching, not overlapping: {state}"
        assert not state.broken
        return [snapshot(scene)]


# --- BounceTest (:37-126) -------------------------------------------------------------------------------------------

RADIUS = 0.05
DROP = 1.0


def rebound(backend, solve, e, snaps):
    with SphereScene(1).uniform(RADIUS, 1) as scene:
        scene.sx = scene.sz = 0.4
        scene.sy = 2
        scene.substeps = 20
        scene.solve = solve
        scene.restitution = e
        scene.x[0] = scene.z[0] = 0.2
        scene.y[0] = f32(RADIUS + DROP)
        scene.start(backend)
        hit = False
        highest = 0.0
        for _ in range(150):
            scene.advance(1).read()
            above = float(scene.y[0]) - RADIUS
            if not hit and scene.v[0] > 0:
                hit = True
            if hit:
                highest = max(highest, above)
                if scene.v[0] < 0 and highest > 0:
                    break
        snaps.append(snapshot(scene))
        return highest


def case_rebound(backend, solve):
    """aBallReboundsToTheSquareOfItsRestitution: it rises to e^2 of its drop, to 1% of the drop."""
    snaps = []
    for e in (0.5, 0.9):
        rose = rebound(backend, solve, e, snaps)
        assert abs(e * e * DROP - rose) <= 0.01 * DROP, f"e = {e}: rose {rose}"
    return snaps


def case_no_bounce(backend, solve):
    """withoutRestitutionABallDoesNotBounce."""
    snaps = []
    assert rebound(backend, solve, 0, snaps) < 0.01 * DROP, "it should stay down"
    return snaps


def case_elastic_collision(backend, solve):
    """anElasticCollisionSwapsTheVelocities: at e = 1 the moving one stops and the other leaves with its speed."""
    with SphereScene(2).uniform(RADIUS, 1) as scene:
        scene.gy = 0
        scene.sx = 2
        scene.sy = scene.sz = 0.4
        scene.substeps = 20
        scene.solve = solve
        scene.restitution = 1
        scene.x[0] = 0.5
        scene.x[1] = 0.8
        scene.y[:] = 0.2
        scene.z[:] = 0.2
        scene.u[0] = 1
        scene.start(backend).advance_seconds(0.5).read()
        assert abs(1 - (float(scene.u[0]) + float(scene.u[1]))) <= 1e-5, "momentum"
        assert abs(scene.u[0]) <= 0.03, "the one that was moving has stopped"
        assert abs(1 - scene.u[1]) <= 0.03, "the one that was at rest has its speed"
        return [snapshot(scene)]


def case_ball_at_rest(backend, solve):
    """aBallAtRestStaysAtRest: a springy ball set down on the floor does not bounce."""
    with SphereScene(1).uniform(RADIUS, 1) as scene:
        scene.sx = scene.sy = scene.sz = 0.4
        scene.substeps = 10
        scene.solve = solve
        scene.restitution = 0.9
        scene.x[0] = scene.z[0] = 0.2
        scene.y[0] = RADIUS
        scene.start(backend).advance_seconds(2).read()
        assert abs(scene.v[0]) < 1e-3, f"speed {scene.v[0]}"
        assert abs(RADIUS - scene.y[0]) <= 1e-4
        return [snapshot(scene)]


# --- SpinTest (:23-95) ----------------------------------------------------------------------------------------------

def case_spin_kept(backend, solve):
    """aSpinIsKeptAndTurnsTheSphereAtItsRate: after 1 s at pi/3 (1, 2, 2) rad/s, turned by pi about (1, 2, 2)/3."""
    with SphereScene(1).uniform(0.1, 1) as scene:
        scene.gy = 0
        scene.x[0] = scene.y[0] = scene.z[0] = 0.5
        rate = f32(math.pi / 3)
        scene.ax[0] = rate
        scene.ay[0] = f32(2 * rate)
        scene.az[0] = f32(2 * rate)
        scene.solve = solve
        scene.start(backend).advance_seconds(1)
        scene.read()
        assert scene.ax[0] == rate and scene.ay[0] == f32(2 * rate) and scene.az[0] == f32(2 * rate)
        q = scene.orientation(0)
        for k, e in enumerate((1 / 3, 2 / 3, 2 / 3, 0)):
            assert abs(e - q[k]) <= 2e-4, f"orientation component {k}"
        assert scene.x[0] == f32(0.5), "spinning does not move it"
        return [snapshot(scene)]


def case_spin_shown(backend, solve):
    """thePictureIsGivenTheOrientationBeforeAndAfterTheStep."""
    with SphereScene(1).uniform(0.1, 1) as scene:
        scene.gy = 0
        scene.x[0] = scene.y[0] = scene.z[0] = 0.5
        scene.ay[0] = 3
        scene.solve = solve
        scene.start(backend).advance(2)
        earlier = scene.shown().copy()
        scene.advance(1)
        shown = scene.shown()
        q = scene.orientation(0)
        for k in range(4):
            assert q[k] == shown[S.TURNED_AFTER + k]
            assert earlier[S.TURNED_AFTER + k] == shown[S.TURNED_BEFORE + k]
        assert abs(0.075 - q[1]) <= 1e-3
        return [snapshot(scene)]


def case_spinning_rest(backend, solve):
    """aSpinningSphereRestsOnTheFloorStillSpinning: no friction, so the floor keeps the spin."""
    with SphereScene(1).uniform(0.1, 2) as scene:
        scene.x[0] = scene.z[0] = 0.5
        scene.y[0] = 0.3
        scene.ax[0] = 10
        scene.solve = solve
        scene.start(backend).advance_seconds(1)
        state = scene.diagnostics()
        assert scene.ax[0] == 10
        assert abs(0.1 - scene.y[0]) <= 1e-6, "resting on the floor"
        assert abs(0.5 * 0.4 * 2 * 0.1 * 0.1 * 100 - state.rotational) <= 1e-6, "the spin's energy"
        assert state.kinetic - state.rotational < 1e-6, f"nothing else moves: {state}"
        return [snapshot(scene)]


# --- PressingTest (:23-96) ------------------------------------------------------------------------------------------

def _pressing(scene, s):
    p = np.zeros(S.PRESSING_WORDS)
    c = [float(scene.x[s]), float(scene.y[s]), float(scene.z[s])]
    r = float(scene.r[s])
    extent = [scene.sx, scene.sy, scene.sz]

    def add(f, n):
        pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
        for k, (i, j) in enumerate(pairs):
            p[S.FLATTENING + k] += f * n[i] * n[j]
        for a in range(3):
            p[S.LEAN + a] += f * n[a]

    for a in range(3):
        for side, depth in enumerate((r - c[a], c[a] + r - extent[a])):
            if depth > 0:
                n = [0.0, 0.0, 0.0]
                n[a] = -1.0 if side == 0 else 1.0
                add(depth / r, n)
    for o in range(scene.n):
        d = [float(scene.x[o]) - c[0], float(scene.y[o]) - c[1], float(scene.z[o]) - c[2]]
        dist = math.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
        reach = r + float(scene.r[o])
        if o != s and dist < reach:
            add((reach - dist) / reach, [d[0] / dist, d[1] / dist, d[2] / dist])
    p[S.TRACE] = p[0] + p[1] + p[2]
    p[S.LEAN_LENGTH] = math.sqrt(p[6] ** 2 + p[7] ** 2 + p[8] ** 2)
    return p


def case_pressing(backend, solve):
    """thePressingIsTheOverlapsTheStepEndedWith: fixed spheres overlapping each other and the walls."""
    with SphereScene(4) as scene:
        at = [(0.05, 0.5, 0.5), (0.2, 0.55, 0.5), (0.25, 0.72, 0.5), (0.5, 0.95, 0.5)]
        radii = [0.1, 0.1, 0.15, 0.1]
        for s in range(4):
            scene.x[s], scene.y[s], scene.z[s] = at[s]
            scene.r[s] = radii[s]
            scene.im[s] = 0
        scene.solve = solve
        scene.start(backend).advance(1)
        earlier = scene.shown().copy()
        scene.advance(1).read()
        shown = scene.shown()
        expected = []
        for s in range(4):
            base = s * S.SHOWN_STRIDE
            e = _pressing(scene, s)
            expected.append(e)
            for k in range(S.LEAN_LENGTH + 1):
                assert abs(e[k] - shown[base + S.PRESSED_AFTER + k]) <= 1e-6, f"sphere {s}, word {k}"
                assert earlier[base + S.PRESSED_AFTER + k] == shown[base + S.PRESSED_BEFORE + k]
        assert abs(0.7094 - expected[0][S.TRACE]) <= 1e-3
        assert abs(-0.3013 - expected[0][S.LEAN]) <= 1e-3
        assert abs(0.2912 - expected[2][S.TRACE]) <= 1e-3
        assert abs(0.5 - expected[3][S.LEAN + 1]) <= 1e-3
        return [snapshot(scene)]


# --- FrictionTest (:14-239) -----------------------------------------------------------------------------------------

def on_the_floor(mu):
    scene = SphereScene(1).uniform(0.1, 1)
    scene.sx = 4
    scene.x[0] = 0.5
    scene.y[0] = 0.1
    scene.z[0] = 0.5
    scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
    scene.mu_static = scene.mu_kinetic = mu
    return scene


def case_slide_to_roll(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aSlidingSphereSettlesIntoRollingAtFiveSevenths."""
    mu, v0 = 0.3, 2.0
    with on_the_floor(mu) as scene:
        scene.u[0] = v0
        scene.start(backend).advance_seconds(0.1)
        scene.read()
        t = 0.1
        assert abs(v0 - mu * G * t - scene.u[0]) <= 1e-2, "slowed by mu g while it slides"
        assert abs(-2.5 * mu * G * t / 0.1 - scene.az[0]) <= 0.1, "spun up by 5 mu g / 2r"
        first = snapshot(scene)
        scene.advance_seconds(0.4)
        state = scene.diagnostics()
        assert abs(5 * v0 / 7 - scene.u[0]) <= 5e-3, f"rolling at 5/7: {state}"
        assert abs(-scene.u[0] / 0.1 - scene.az[0]) <= 1e-2, "omega = -v / r"
        assert abs(0.1 - scene.y[0]) <= 1e-5, "on the floor"
        assert abs(scene.ax[0]) <= 1e-6 and abs(scene.ay[0]) <= 1e-6
        return [first, snapshot(scene)]


def case_slope(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """onASlopeASphereRollsWithEnoughFrictionAndSlidesWithout (gravity tilted by 20 degrees)."""
    theta = math.radians(20)
    t = 0.5
    snaps = []
    with on_the_floor(0.5) as rolling:
        rolling.x[0] = 0.2
        rolling.gx = G * math.sin(theta)
        rolling.gy = -G * math.cos(theta)
        rolling.start(backend).advance_seconds(t)
        rolling.read()
        assert abs(5.0 / 7 * G * math.sin(theta) * t - rolling.u[0]) <= 1e-2, "rolling at 5/7 g sin theta"
        assert abs(-rolling.u[0] / 0.1 - rolling.az[0]) <= 1e-2, "without slipping"
        snaps.append(snapshot(rolling))
    mu = 0.05
    with on_the_floor(mu) as sliding:
        sliding.x[0] = 0.2
        sliding.gx = G * math.sin(theta)
        sliding.gy = -G * math.cos(theta)
        sliding.start(backend).advance_seconds(t)
        sliding.read()
        assert abs(G * (math.sin(theta) - mu * math.cos(theta)) * t - sliding.u[0]) <= 1e-2
        assert abs(-2.5 * mu * G * math.cos(theta) * t / 0.1 - sliding.az[0]) <= 0.05
        snaps.append(snapshot(sliding))
    return snaps


def glancing(mu):
    scene = SphereScene(2).uniform(0.1, 1)
    scene.gy = 0
    scene.sx = 4
    scene.im[1] = f32(1 / 3)
    scene.x[0] = 1
    scene.x[1] = 1.5
    scene.y[0] = 0.5
    scene.y[1] = 0.55
    scene.z[:] = 0.5
    scene.u[0] = 2
    scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
    scene.mu_static = scene.mu_kinetic = mu
    return scene


def case_glancing(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aGlancingCollisionKeepsMomentumAndAngularMomentumToFirstOrder."""
    frictionless, with_friction = [0.0, 0.0], [0.0, 0.0]
    snaps = []
    for run in range(2):
        for mu in (0.0, 0.5):
            with glancing(mu) as scene:
                scene.substeps = 10 << run
                start = S.diagnostics(scene.x, scene.y, scene.z, scene.u, scene.v, scene.w, scene.ax, scene.ay,
                                      scene.az, scene.r, scene.im, 0, scene.sx, scene.sy, scene.sz)
                scene.start(backend).advance_seconds(0.5)
                end = scene.diagnostics()
                for k in range(3):
                    assert abs(start.momentum[k] - end.momentum[k]) <= 1e-5, f"momentum {k}: {end}"
                change = abs(end.angular[2] - start.angular[2])
                assert abs(end.angular[0]) <= 1e-6
                assert abs(start.angular[1] - end.angular[1]) <= 1e-6
                if mu == 0:
                    frictionless[run] = change
                    assert end.rotational == 0, f"without friction nothing spins: {end}"
                else:
                    with_friction[run] = change
                    assert abs(scene.az[0]) > 1 and abs(scene.az[1]) > 0.1, "friction spun them"
                    assert end.kinetic < start.kinetic, f"friction only takes energy: {end}"
                snaps.append(snapshot(scene))
        assert with_friction[run] <= frictionless[run]
    assert with_friction[1] < 0.6 * with_friction[0], "first order: halved with the substep"
    assert with_friction[0] < 1.5e-3, "small at 10 substeps"
    return snaps


def case_wedged_on_slope(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aSphereWedgedOnASlopeRests: against a fixed sphere below it on a 20 degree slope."""
    theta = math.radians(20)
    with SphereScene(2).uniform(0.03, 0.1) as scene:
        scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
        scene.mu_static = scene.mu_kinetic = 0.5
        scene.sx = scene.sy = scene.sz = 0.5
        scene.gx = G * math.sin(theta)
        scene.gy = -G * math.cos(theta)
        scene.x[0] = 0.2
        scene.x[1] = 0.26
        scene.y[:] = 0.03
        scene.z[:] = 0.25
        scene.im[1] = 0
        scene.start(backend).advance_seconds(1)
        scene.read()
        assert abs(scene.az[0]) < 1.5e-4, f"not spinning in place: {scene.az[0]}"
        assert math.hypot(scene.u[0], scene.v[0]) < 5e-6, f"still: {scene.u[0]}, {scene.v[0]}"
        assert abs(0.2 - scene.x[0]) <= 1e-5, "where it was put"
        return [snapshot(scene)]


def case_pocket(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aSphereInAPocketStopsSpinning: set spinning in the pocket of three fixed spheres."""
    r = 0.03
    with SphereScene(4).uniform(r, 0.1) as scene:
        scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
        scene.mu_static = scene.mu_kinetic = 0.5
        scene.sx = scene.sy = scene.sz = 0.5
        c = 0.25
        for k in range(3):
            angle = 2 * math.pi * k / 3
            scene.x[k] = f32(c + 2 * r / math.sqrt(3) * math.cos(angle))
            scene.z[k] = f32(c + 2 * r / math.sqrt(3) * math.sin(angle))
            scene.y[k] = f32(r)
            scene.im[k] = 0
        scene.x[3] = scene.z[3] = f32(c)
        scene.y[3] = f32(r + 2 * r * math.sqrt(2.0 / 3))
        scene.ax[3], scene.ay[3], scene.az[3] = 1, 2, 3
        scene.start(backend).advance_seconds(1)
        scene.read()
        spin = math.sqrt(float(scene.ax[3]) ** 2 + float(scene.ay[3]) ** 2 + float(scene.az[3]) ** 2)
        assert spin < 2e-3, f"stopped spinning: {spin} rad/s"
        return [snapshot(scene)]


def case_column_with_friction(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aColumnStillRestsWithFriction: a column of ten rests."""
    with SphereScene(10).uniform(0.05, 1) as scene:
        for k in range(10):
            scene.x[k] = scene.z[k] = 0.5
            scene.y[k] = f32(f32(0.05) + f32(0.1) * f32(k))
        scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
        scene.mu_static = scene.mu_kinetic = 0.5
        scene.start(backend).advance_seconds(2)
        state = scene.diagnostics()
        assert state.kinetic < 1e-6, f"at rest: {state}"
        assert state.max_overlap < 0.05, f"standing: {state}"
        assert abs(scene.x[9] - 0.5) < 1e-4, "upright"
        return [snapshot(scene)]


# --- RollingTest (:14-88) -------------------------------------------------------------------------------------------

def rolling(v0, mu_rolling):
    scene = SphereScene(1).uniform(0.1, 1)
    scene.sx = 6
    scene.x[0] = 0.5
    scene.y[0] = 0.1
    scene.z[0] = 0.5
    scene.u[0] = f32(v0)
    scene.az[0] = f32(-v0 / 0.1)
    scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
    scene.mu_static = scene.mu_kinetic = 0.5
    scene.mu_rolling = mu_rolling
    return scene


def case_rolling_resistance(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aRollingSphereSlowsAtFiveSeventhsOfMuGAndStops."""
    mu = 0.1
    with rolling(1, mu) as scene:
        scene.start(backend).advance_seconds(0.5)
        scene.read()
        expected = 1 - 5.0 / 7 * mu * G * 0.5
        assert abs(expected - scene.u[0]) <= 1e-2, "slowed at 5/7 mu_r g"
        assert abs(-scene.u[0] / 0.1 - scene.az[0]) <= 5e-2, "still rolling"
        scene.advance_seconds(1.5)
        scene.read()
        assert abs(scene.u[0]) < 1e-4, f"stopped: {scene.u[0]}"
        assert abs(scene.az[0]) < 1e-3, f"not turning: {scene.az[0]}"
        stopped = float(scene.x[0])
        scene.advance_seconds(1)
        scene.read()
        assert abs(stopped - scene.x[0]) <= 1e-5, "and stays where it stopped"
        return [snapshot(scene)]


def case_rolls_on(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """withoutItASphereRollsOn."""
    with rolling(1, 0) as scene:
        scene.start(backend).advance_seconds(1)
        scene.read()
        assert abs(1 - scene.u[0]) <= 1e-3
        assert abs(-10 - scene.az[0]) <= 1e-2
        return [snapshot(scene)]


def case_twist_stops(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aSphereSpinningOnTheFloorStops: rolling resistance takes twisting too."""
    with rolling(0, 0.1) as scene:
        scene.ay[0] = 5
        scene.start(backend).advance_seconds(0.1)
        scene.read()
        assert abs(5 - 0.1 * G / (S.INERTIA * 0.1) * 0.1 - scene.ay[0]) <= 5e-2
        scene.advance_seconds(0.5)
        scene.read()
        assert abs(scene.ay[0]) < 1e-3, f"stopped: {scene.ay[0]}"
        return [snapshot(scene)]


# --- GridTest (:26-66) ----------------------------------------------------------------------------------------------

def crowd():
    n = 600
    scene = SphereScene(n)
    scene.sx, scene.sy, scene.sz = 0.6, 0.4, 0.5
    rnd = JavaRandom(5)
    for k in range(n):
        scene.r[k] = f32(0.02 + 0.03 * rnd.next_double())
        scene.im[k] = f32(1 / (0.1 + rnd.next_double()))
        scene.x[k] = f32(-0.05 + 0.7 * rnd.next_double())
        scene.y[k] = f32(0.4 * rnd.next_double())
        scene.z[k] = f32(0.5 * rnd.next_double())
    return scene


def case_grid_finds_every_pair(backend, solve=S.JACOBI):
    """theGridFindsWhatEveryPairFinds: one step from the same crowded state, agreeing to 1e-5 m."""
    pairs, grid = crowd(), crowd()
    grid.grid = True
    with pairs, grid:
        pairs.start(backend).advance(1).read()
        grid.start(backend).advance(1).read()
        worst = max(float(np.max(np.abs(pairs.x - grid.x))), float(np.max(np.abs(pairs.y - grid.y))),
                    float(np.max(np.abs(pairs.z - grid.z))))
        assert worst < 1e-5, f"the searches disagree by {worst} m"
        return [snapshot(pairs), snapshot(grid)]


# --- PileTest (:33-101) ---------------------------------------------------------------------------------------------

def case_dropped_pile(backend, grid, solve, mu, seconds=3):
    """aDroppedPileStaysInsideApartAndLosesEnergy: 125 spheres in a loose lattice, three seconds."""
    side = 5
    with SphereScene(side ** 3).uniform(0.03, 0.1) as scene:
        scene.sx = scene.sz = 0.4
        scene.sy = 1
        scene.substeps = 20
        scene.grid = grid
        scene.solve = solve
        scene.mu_static = scene.mu_kinetic = mu
        rnd = JavaRandom(11)
        k = 0
        for i in range(side):
            for j in range(side):
                for l in range(side):
                    scene.x[k] = f32(0.07 + 0.065 * i + 0.005 * rnd.next_double())
                    scene.y[k] = f32(0.2 + 0.07 * j)
                    scene.z[k] = f32(0.07 + 0.065 * l + 0.005 * rnd.next_double())
                    k += 1
        start = S.diagnostics(scene.x, scene.y, scene.z, scene.u, scene.v, scene.w, scene.ax, scene.ay, scene.az,
                              scene.r, scene.im, scene.gy, scene.sx, scene.sy, scene.sz)
        scene.start(backend)
        worst = 0.0
        snaps = []
        for second in range(seconds):
            state = scene.advance_seconds(1).diagnostics()
            assert not state.broken, f"non-finite after {second + 1} s"
            assert state.max_wall < 1e-5, f"outside the box: {state}"
            worst = max(worst, state.max_overlap)
            assert state.kinetic + state.potential < start.kinetic + start.potential, f"energy grew: {state}"
            snaps.append(snapshot(scene))
        assert worst < 0.2, f"spheres passed into each other by {worst} of a radius"
        return snaps


def friction_pile():
    side = 7
    scene = SphereScene(side ** 3).uniform(0.03, 0.1)
    scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
    scene.mu_static = scene.mu_kinetic = 0.5
    scene.sx = scene.sz = 0.08 + 0.06 * side
    scene.sy = 0.5 + 0.07 * side
    rnd = JavaRandom(7)
    k = 0
    for i in range(side):
        for j in range(side):
            for l in range(side):
                scene.x[k] = f32(0.07 + 0.06 * i + 0.005 * rnd.next_double())
                scene.y[k] = f32(0.3 + 0.07 * j)
                scene.z[k] = f32(0.07 + 0.06 * l + 0.005 * rnd.next_double())
                k += 1
    return scene


def case_friction_pile_rests(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """aPileWithFrictionComesToRest: 343 spheres at mu 0.5 and 10 substeps settle within 4 s and then rest."""
    with friction_pile() as scene:
        scene.start(backend).advance_seconds(4)
        settled = scene.diagnostics().potential
        later = scene.advance_seconds(2).diagnostics()
        creep = (settled - later.potential) / 2
        assert creep < 5e-3, f"still creeping, {creep} J a second: {later}"
        assert later.kinetic < 1e-4, f"at rest: {later}"
        return [snapshot(scene)]


# --- UntilDoneTest (:27-68) -----------------------------------------------------------------------------------------

ENOUGH = S.CYCLE - 1


def until_done_pile():
    n = 300
    scene = SphereScene(n)
    scene.sx = scene.sz = 0.5
    scene.sy = 1
    scene.substeps = 10
    scene.solve = S.GAUSS_SEIDEL_BY_CONTACT
    rnd = JavaRandom(5)
    for k in range(n):
        scene.r[k] = f32(0.02 + 0.015 * rnd.next_double())
        scene.im[k] = f32(1 / (0.05 + 0.2 * rnd.next_double()))
        scene.x[k] = f32(0.05 + 0.4 * rnd.next_double())
        scene.y[k] = f32(0.05 + 0.3 * rnd.next_double())
        scene.z[k] = f32(0.05 + 0.4 * rnd.next_double())
    return scene


def case_until_done(backend, solve=S.GAUSS_SEIDEL_BY_CONTACT):
    """untilDoneIsEnoughRoundsAndLeavesNothingUnsolved: the same state to the bit as ENOUGH fixed rounds."""
    with until_done_pile() as scene:
        scene.fixed_rounds = True
        scene.rounds = ENOUGH
        scene.start(backend).advance_seconds(0.25).read()
        fixed = [scene.x.copy(), scene.y.copy(), scene.z.copy(), scene.v.copy()]
        assert scene.contact_count()[S.MISSED] == 0, "the fixed solve had enough rounds"
        first = snapshot(scene)
    with until_done_pile() as scene:
        scene.start(backend).advance_seconds(0.25).read()
        assert scene.most_rounds <= ENOUGH, f"a pass needed {scene.most_rounds} rounds"
        assert scene.unlisted == 0
        for a, b in zip(fixed, [scene.x, scene.y, scene.z, scene.v]):
            assert np.array_equal(a, b)
        return [first, snapshot(scene)]


EVERY_SOLVE_CASES = [case_fall, case_rest_on_floor, case_inelastic_collision, case_rebound, case_no_bounce,
                     case_elastic_collision, case_ball_at_rest, case_spin_kept, case_spin_shown, case_spinning_rest,
                     case_pressing]
FRICTION_CASES = [case_slide_to_roll, case_slope, case_glancing, case_wedged_on_slope, case_pocket,
                  case_column_with_friction, case_rolling_resistance, case_rolls_on, case_twist_stops]
