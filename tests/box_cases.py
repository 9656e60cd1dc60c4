"""Step-level known-answer cases of the reference's box tests, each a function of the backend.

Restated from vexelray-sim-rigid-core/src/test/java/dev/vexelray/sim/rigid/box/: BoxBroadTest.java,
BoxFreeTest.java, BoxStackTest.java, BoxWallTest.java, BoxSphereTest.java and BoxShowTest.java, with the reference's
tolerances. test_oracle_box.py runs them on the oracle (pinning it); test_gpu_box.py runs them on the CUDA library.
"""
import math

import numpy as np

from box_scene import BoxScene
from java_random import JavaRandom
from vxr import boxes as B

G = 9.81
HX, HY, HZ = 0.05, 0.1, 0.2


# --- BoxBroadTest.theGridFindsWhatEveryPairFinds (:35-101) -------------------------------------------------------

def broad_fixture():
    n = 150
    rnd = JavaRandom(23)
    scene = BoxScene(n)
    widest = 0.0
    for s in range(n):
        half = [0.02 + 0.06 * rnd.next_double() for _ in range(3)]
        widest = max(widest, math.sqrt(half[0] * half[0] + half[1] * half[1] + half[2] * half[2]))
        axis = [rnd.next_double() - 0.5 for _ in range(3)]
        length = math.sqrt(axis[0] ** 2 + axis[1] ** 2 + axis[2] ** 2)
        angle = 4 * rnd.next_double()
        sn = math.sin(angle / 2) / length
        q = [axis[0] * sn, axis[1] * sn, axis[2] * sn, math.cos(angle / 2)]
        pos = [0.1 + 0.8 * rnd.next_double() for _ in range(3)]
        scene.x[s], scene.y[s], scene.z[s] = pos
        scene.half[:, s] = half
        scene.q[:, s] = q
    scene.widest = widest
    scene.gy = 0.0
    scene.dt = 1e-3
    scene.substeps = 1
    scene.passes = 1
    scene.margin = 0.005
    return scene


def every_pair_touching(scene, backend):
    """Every pair collided alone (BoxBroadTest.EveryPair): {(a, b): points}."""
    n = scene.n
    list_ = [(a, b) for a in range(n) for b in range(a + 1, n)]
    pairs = np.array(list_, dtype=np.int32).reshape(-1)
    f = [scene.x, scene.y, scene.z, scene.u, scene.v, scene.w, scene.l[0], scene.l[1], scene.l[2], scene.q[0],
         scene.q[1], scene.q[2], scene.q[3], scene.im, scene.half[0], scene.half[1], scene.half[2], scene.shape]
    bits = B.params(1e-3, 0, 0, 0, 1, 1, 1, 0, 0, scene.margin)
    if backend == "oracle":
        from oracle.box import collide
        m = collide(f, bits, pairs)
    else:
        from vxr.box_simulation import collide_pairs
        m = collide_pairs(f, bits, pairs)
    out = {}
    for p, (a, b) in enumerate(list_):
        c = int(m[p * 40 + B.COUNT])
        if c > 0:
            out[(a, b)] = c
    return out


def case_grid_finds_every_pair(backend):
    scene = broad_fixture()
    scene.start(backend)
    scene.advance(1)
    grid = {(a, b): c for a, b, c in scene.world.touching_pairs()}
    every = every_pair_touching(scene, backend)
    assert len(every) > 100
    assert scene.unlisted == 0
    assert grid == every
    scene.close()
    return grid


# --- BoxFreeTest ---------------------------------------------------------------------------------------------------

def case_free_fall(backend):
    scene = BoxScene(1).uniform(HX, HY, HZ, 1)
    scene.sy = 20
    scene.x[0] = scene.z[0] = 0.5
    scene.y[0] = 8
    scene.start(backend).advance_seconds(0.5).read()
    substeps = 30 * scene.substeps
    h = scene.dt / scene.substeps
    y, vy = 8.0, 0.0
    for _ in range(substeps):
        vy += h * scene.gy
        y += h * vy
    assert abs(vy - scene.v[0]) <= 1e-5
    assert abs(y - scene.y[0]) <= 1e-5
    assert scene.q[3][0] == 1
    scene.close()


def case_stable_spin(backend, seconds=10.0):
    for axis in (0, 2):
        scene = BoxScene(1).uniform(HX, HY, HZ, 1)
        scene.gy = 0
        scene.x[0] = scene.y[0] = scene.z[0] = 0.5
        [scene.ax, scene.ay, scene.az][axis][0] = 5
        scene.start(backend).advance_seconds(seconds).read()
        own = scene.own_spin(0)
        for a in range(3):
            assert abs((5 if a == axis else 0) - own[a]) <= 1e-4
        angle = 2 * math.atan2(float(scene.q[axis][0]), float(scene.q[3][0]))
        expected = math.remainder(5 * seconds, 2 * math.pi)
        assert abs(math.remainder(angle - expected, 2 * math.pi)) <= 1e-3
        scene.close()


def tumbling():
    scene = BoxScene(1).uniform(HX, HY, HZ, 2)
    scene.gy = 0
    scene.sx = scene.sy = scene.sz = 100
    scene.x[0] = scene.y[0] = scene.z[0] = 50
    scene.u[0] = 1
    scene.ax[0], scene.ay[0], scene.az[0] = 1, 2, 3
    return scene


def case_tumble_keeps_momentum_and_energy(backend, seconds=10.0):
    scene = tumbling()
    before = scene.start(backend).diagnostics()
    scene.advance_seconds(seconds)
    after = scene.diagnostics()
    length = math.sqrt(sum(c * c for c in before.angular))
    drift = math.sqrt(sum((a - b) ** 2 for a, b in zip(after.angular, before.angular))) / length
    energy = abs(after.kinetic - before.kinetic) / before.kinetic
    assert drift == 0, f"angular momentum moved by {drift}"
    assert energy < 1e-6, f"energy moved by {energy}"
    assert abs(scene.own_spin(0)[1]) > 0.1
    scene.close()


# --- BoxStackTest ---------------------------------------------------------------------------------------------------

def case_head_on(backend):
    scene = BoxScene(2).uniform(0.05, 0.05, 0.05, 1)
    scene.gy = 0
    scene.sx = scene.sy = scene.sz = 2
    scene.x[0], scene.x[1] = 0.8, 1.2
    scene.y[:] = 1
    scene.z[:] = 1
    scene.u[0], scene.u[1] = 1, -1
    scene.start(backend).advance_seconds(0.5)
    state = scene.diagnostics()
    assert abs(state.momentum[0]) <= 1e-6
    assert abs(scene.u[0]) <= 1e-3 and abs(scene.u[1]) <= 1e-3
    assert abs(0.1 - (float(scene.x[1]) - float(scene.x[0]))) <= 1e-3
    scene.close()


def column_scene(n):
    scene = BoxScene(n).uniform(0.05, 0.05, 0.05, 1)
    scene.sx = scene.sz = 1
    scene.sy = 0.11 * n + 0.5
    for k in range(n):
        scene.x[k] = scene.z[k] = 0.5
        scene.y[k] = 0.05 + 0.101 * k
    scene.mu_static = scene.mu_kinetic = 0.5
    return scene


def case_column(backend, n=10, most_drift=1e-3, most_energy=1e-6, seconds=3.0):
    scene = column_scene(n)
    scene.start(backend).advance_seconds(seconds)
    state = scene.diagnostics()
    drift = math.hypot(float(scene.x[n - 1]) - 0.5, float(scene.z[n - 1]) - 0.5)
    assert drift < most_drift
    assert state.kinetic < most_energy, state.kinetic
    assert scene.unplaced == 0
    scene.close()


def pile_scene(side):
    n = side ** 3
    scene = BoxScene(n).uniform(0.04, 0.04, 0.04, 0.5)
    scene.mu_static = scene.mu_kinetic = 0.5
    scene.sx = scene.sz = 0.1 * side + 0.4
    scene.sy = 0.1 * side + 1.5
    rnd = JavaRandom(7)
    k = 0
    for i in range(side):
        for j in range(side):
            for l_ in range(side):
                scene.x[k] = 0.25 + 0.1 * i + 0.02 * rnd.next_double()
                scene.y[k] = 0.3 + 0.1 * j
                scene.z[k] = 0.25 + 0.1 * l_ + 0.02 * rnd.next_double()
                axis = [rnd.next_double() - 0.5 for _ in range(3)]
                length = math.sqrt(axis[0] ** 2 + axis[1] ** 2 + axis[2] ** 2)
                angle = 0.6 * rnd.next_double()
                sn = math.sin(angle / 2) / length
                for a in range(3):
                    scene.q[a][k] = axis[a] * sn
                scene.q[3][k] = math.cos(angle / 2)
                k += 1
    return scene


def case_pile(backend, side=7, most_energy=1e-6, most_depth=1e-3, **kw):
    """BoxStackTest.pile (:184-232): 343 cubes dropped, resting after 4 s."""
    scene = pile_scene(side)
    scene.start(backend, **kw).advance_seconds(3)
    scene.advance_seconds(1)
    state = scene.diagnostics()
    deepest = scene.deepest()
    assert state.kinetic < most_energy, state.kinetic
    assert deepest < most_depth, deepest
    assert scene.unplaced == 0
    assert scene.unlisted == 0
    scene.close()


# --- BoxWallTest ----------------------------------------------------------------------------------------------------

def axis_of(scene, s, k):
    unit = [0.0, 0.0, 0.0]
    unit[k] = 1.0
    return B.rotate([float(c) for c in scene.q[:, s]], unit)


def tilt_of(unit):
    return math.asin(min(1.0, math.hypot(unit[0], unit[2])))


def case_flat_rests_flat(backend):
    scene = BoxScene(1).uniform(0.1, 0.05, 0.1, 1)
    scene.x[0] = scene.z[0] = 0.5
    scene.y[0] = 0.06
    scene.mu_static = scene.mu_kinetic = 0.5
    scene.start(backend).advance_seconds(2)
    state = scene.diagnostics()
    assert tilt_of(axis_of(scene, 0, 1)) < 1e-4
    assert abs(0.05 - scene.y[0]) <= 1e-4
    assert abs(0.5 - scene.x[0]) <= 1e-4 and abs(0.5 - scene.z[0]) <= 1e-4
    assert state.kinetic < 1e-6
    scene.close()


def on_a_slope(degrees, mu):
    scene = BoxScene(1).uniform(0.1, 0.05, 0.1, 1)
    theta = math.radians(degrees)
    scene.gx = G * math.sin(theta)
    scene.gy = -G * math.cos(theta)
    scene.sx = 10
    scene.x[0] = 1
    scene.z[0] = 0.5
    scene.y[0] = 0.05
    scene.mu_static = scene.mu_kinetic = mu
    return scene


def case_slope_holds(backend):
    scene = on_a_slope(20, 0.5)
    scene.start(backend).advance_seconds(1).read()
    settled = float(scene.x[0])
    scene.advance_seconds(2).read()
    assert abs(1 - settled) <= 1e-5
    assert abs(settled - float(scene.x[0])) <= 1e-5
    assert abs(float(scene.u[0])) <= 1e-5
    scene.close()


def case_slope_slides(backend):
    theta = math.radians(30)
    scene = on_a_slope(30, 0.3)
    scene.start(backend).advance_seconds(0.5).read()
    early = float(scene.u[0])
    scene.advance_seconds(0.5).read()
    rate = (float(scene.u[0]) - early) / 0.5
    expected = G * (math.sin(theta) - 0.3 * math.cos(theta))
    assert abs(expected - rate) <= 0.01 * expected
    assert tilt_of(axis_of(scene, 0, 1)) < 1e-3
    scene.close()


# --- BoxSphereTest --------------------------------------------------------------------------------------------------

def case_ball_rests_on_box(backend):
    scene = BoxScene(2).uniform(0.05, 0.05, 0.05, 1)
    scene.sphere(1, 0.05)
    scene.im[1] = 2
    scene.mu_static = scene.mu_kinetic = 0.5
    scene.x[:] = 0.5
    scene.z[:] = 0.5
    scene.y[0] = 0.05
    scene.y[1] = 0.151
    scene.start(backend).advance_seconds(2)
    state = scene.diagnostics()
    assert abs(0.15 - scene.y[1]) <= 5e-4
    assert math.hypot(float(scene.x[1]) - 0.5, float(scene.z[1]) - 0.5) < 1e-4
    assert state.kinetic < 1e-6
    scene.close()


def case_sliding_ball_rolls(backend):
    scene = BoxScene(2).uniform(1.8, 0.05, 0.3, 1)
    scene.sphere(1, 0.05)
    scene.im[0] = 0
    scene.mu_static = scene.mu_kinetic = 0.3
    scene.sx = 4
    scene.sz = 1
    scene.x[0] = 2
    scene.y[0] = 0.05
    scene.z[:] = 0.5
    scene.x[1] = 0.4
    scene.y[1] = 0.15
    scene.u[1] = 2
    scene.start(backend).advance_seconds(1)
    scene.read()
    rolling = 2 * 5.0 / 7
    assert abs(rolling - scene.u[1]) <= 0.01 * rolling
    assert abs(-rolling / 0.05 - scene.az[1]) <= 0.01 * rolling / 0.05
    assert abs(0.15 - scene.y[1]) <= 5e-4
    scene.close()


def case_rolling_resistance(backend):
    for on_slab in (False, True):
        n = 2 if on_slab else 1
        scene = BoxScene(n).uniform(1.8, 0.05, 0.3, 1)
        ball = n - 1
        scene.sphere(ball, 0.05)
        scene.mu_static = scene.mu_kinetic = 0.5
        scene.mu_rolling = 0.1
        scene.sx = 4
        scene.sz = 1
        if on_slab:
            scene.im[0] = 0
            scene.x[0] = 2
            scene.y[0] = 0.05
            scene.z[0] = 0.5
        scene.x[ball] = 0.4
        scene.y[ball] = 0.15 if on_slab else 0.05
        scene.z[ball] = 0.5
        scene.u[ball] = 1
        scene.az[ball] = -20
        scene.start(backend).advance_seconds(0.5)
        scene.read()
        expected = 1 - 0.5 * 5.0 / 7 * 0.1 * G
        assert abs(expected - scene.u[ball]) <= 1e-2
        assert abs(-float(scene.u[ball]) / 0.05 - float(scene.az[ball])) <= 0.2
        scene.close()


def case_ball_into_box(backend):
    scene = BoxScene(2).uniform(0.05, 0.05, 0.05, 1)
    scene.sphere(0, 0.05)
    scene.gy = 0
    scene.sx = scene.sy = scene.sz = 2
    scene.x[0] = 0.7
    scene.x[1] = 1
    scene.y[:] = 1
    scene.z[:] = 1
    scene.u[0] = 2
    scene.start(backend).advance_seconds(0.5)
    state = scene.diagnostics()
    assert abs(2 - state.momentum[0]) <= 1e-6
    assert abs(1 - scene.u[0]) <= 1e-2 and abs(1 - scene.u[1]) <= 1e-2
    scene.close()


def mixed_pile_scene(side=4):
    n = 2 * side ** 3
    scene = BoxScene(n).uniform(0.04, 0.04, 0.04, 0.5)
    scene.mu_static = scene.mu_kinetic = 0.5
    scene.mu_rolling = 0.3
    scene.sx = scene.sz = 1
    scene.sy = 2.5
    rnd = JavaRandom(3)
    k = 0
    for i in range(side):
        for j in range(2 * side):
            for l_ in range(side):
                if k % 2 == 0:
                    scene.sphere(k, 0.04)
                scene.x[k] = 0.35 + 0.1 * i + 0.02 * rnd.next_double()
                scene.y[k] = 0.3 + 0.1 * j
                scene.z[k] = 0.35 + 0.1 * l_ + 0.02 * rnd.next_double()
                k += 1
    return scene


def case_mixed_pile_rests(backend):
    """BoxSphereTest.aMixedPileRests (:169-210)."""
    scene = mixed_pile_scene()
    scene.start(backend).advance_seconds(4)
    state = scene.diagnostics()
    assert state.kinetic < 1e-5, state.kinetic
    assert scene.deepest() < 2e-3
    assert scene.unplaced == 0 and scene.unlisted == 0
    scene.close()


# --- BoxShowTest.thePictureIsGivenEachStepAndTheOneBefore (:184-220) -------------------------------------------------

def case_show(backend):
    scene = BoxScene(2).uniform(0.05, 0.1, 0.15, 1)
    scene.x[0] = scene.y[0] = scene.z[0] = 0.5
    scene.ax[0], scene.ay[0], scene.az[0] = 1, 2, 3
    scene.x[1], scene.y[1], scene.z[1] = 0.2, 0.1, 0.8
    scene.im[1] = 0
    scene.half[2][1] = 0.05
    scene.start(backend).advance(2)
    earlier = scene.world.shown().copy()
    scene.advance(1).read()
    shown = scene.world.shown()
    at = [scene.x, scene.y, scene.z]
    for s in range(2):
        base = s * B.SHOWN_STRIDE
        for a in range(3):
            assert at[a][s] == shown[base + B.CENTRE_AFTER + a]
            assert earlier[base + B.CENTRE_AFTER + a] == shown[base + B.CENTRE_BEFORE + a]
            assert scene.half[a][s] == shown[base + B.HALF + a]
        for k in range(4):
            assert scene.q[k][s] == shown[base + B.TURNED_AFTER + k]
            assert earlier[base + B.TURNED_AFTER + k] == shown[base + B.TURNED_BEFORE + k]
    assert shown[B.CENTRE_AFTER + 1] < shown[B.CENTRE_BEFORE + 1]
    assert shown[B.TURNED_AFTER] != shown[B.TURNED_BEFORE]
    scene.close()
