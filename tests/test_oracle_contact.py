"""Pins the oracle's narrow phase to the reference's own known-answer tests.

Restates vexelray-sim-rigid-core/src/test/java/dev/vexelray/sim/rigid/box/BoxContactTest.java: 11 hand-worked box
cases, 6 sphere cases and 500 random pairs (java.util.Random(19)), with the reference's tolerances (normals to
2e-6, points to 1e-5, depths to 2e-6). The same cases run against the CUDA kernel in test_gpu_box.py.
"""
import math

import numpy as np
import pytest

from java_random import JavaRandom
from vxr import boxes as B

SLAB = (0.3, 0.1, 0.3)
CUBE = (0.1, 0.1, 0.1)
IDENTITY = (0.0, 0.0, 0.0, 1.0)
R2 = math.sqrt(2)
CLOSE = 2e-6


class Solid:
    def __init__(self, centre, half, q, shape=B.BOX_SHAPE):
        self.centre, self.half, self.q, self.shape = centre, half, q, shape

    def world(self, m, at):
        own = [float(m[at]), float(m[at + 1]), float(m[at + 2])]
        t = B.rotate(self.q, own)
        return [self.centre[0] + t[0], self.centre[1] + t[1], self.centre[2] + t[2]]


def box(x, y, z, half, q):
    return Solid((x, y, z), half, q)


def ball(x, y, z, r):
    return Solid((x, y, z), (r, r, r), IDENTITY, B.SPHERE_SHAPE)


def axis_angle(x, y, z, angle):
    length = math.sqrt(x * x + y * y + z * z)
    s = math.sin(angle / 2) / length
    return (x * s, y * s, z * s, math.cos(angle / 2))


def fields_of(solids):
    """The 18 per-body fields (x..shape) as f32 arrays, as BoxContactTest.collide writes them."""
    n = len(solids)
    f = [np.zeros(n, np.float32) for _ in range(18)]
    f[12][:] = 1  # qw
    for s, b in enumerate(solids):
        for a in range(3):
            f[a][s] = b.centre[a]
            f[14 + a][s] = b.half[a]
        for k in range(4):
            f[9 + k][s] = b.q[k]
        f[17][s] = b.shape
    return f


def collide_backend(backend, margin, *solids):
    """Manifolds of pairs (solids[0], solids[1]), (solids[2], solids[3]) ... on a backend."""
    pairs = np.arange(len(solids), dtype=np.int32)
    bits = B.params(1e-3, 0, 0, 0, 1, 1, 1, 0, 0, margin)
    f = fields_of(solids)
    if backend == "oracle":
        from oracle.box import collide
        return collide(f, bits, pairs)
    from vxr.box_simulation import collide_pairs
    return collide_pairs(f, bits, pairs)


class Contact:
    def __init__(self, m, first, second):
        self.m, self.first, self.second = m, first, second

    def face(self, axis, nx, ny, nz):
        assert self.m[B.AXIS] == axis, f"the axis that won: {self.m[B.AXIS]}"
        self.normal(nx, ny, nz)

    def normal(self, nx, ny, nz):
        for a, v in enumerate((nx, ny, nz)):
            assert abs(v - self.m[B.NORMAL + a]) <= CLOSE, f"normal {a}: {self.m[B.NORMAL + a]}"

    def points(self, depth, on_second):
        n = [float(self.m[B.NORMAL + a]) for a in range(3)]
        on_first = [[p[a] + depth * n[a] for a in range(3)] for p in on_second]
        self.points_on(depth, on_first, on_second)

    def points_on(self, depth, on_first, on_second):
        count = int(self.m[B.COUNT])
        found = []
        for k in range(count):
            at = B.POINTS + k * B.POINT_WORDS
            found.append((self.first.world(self.m, at + B.ANCHOR_FIRST),
                          self.second.world(self.m, at + B.ANCHOR_SECOND), float(self.m[at + B.DEPTH])))
        assert len(on_first) == count, f"points: {found}"
        used = [False] * count
        for e in range(len(on_first)):
            matched = False
            for k in range(count):
                if used[k] or matched:
                    continue
                if near(found[k][0], on_first[e]) and near(found[k][1], on_second[e]):
                    used[k] = matched = True
                    assert abs(depth - found[k][2]) <= CLOSE, f"depth of {on_second[e]}: {found[k][2]}"
            assert matched, f"no point at {on_first[e]} / {on_second[e]} in {found}"


def near(p, q):
    return all(abs(p[a] - q[a]) < 1e-5 for a in range(3))


def corners(hx, hy, hz, y):
    return [[hx, y, hz], [hx, y, -hz], [-hx, y, hz], [-hx, y, -hz]]


# Every case below is one of BoxContactTest's, by the same name; BACKENDS lets the GPU parity file reuse them.
def case_boxes_apart(backend):
    m = collide_backend(backend, 0, box(0, 0, 0, CUBE, IDENTITY), box(0.25, 0, 0, CUBE, IDENTITY))
    assert m[B.COUNT] == 0


def case_cube_on_slab(backend):
    slab, cube = box(0, 0, 0, SLAB, IDENTITY), box(0, 0.19, 0, CUBE, IDENTITY)
    c = Contact(collide_backend(backend, 0, slab, cube), slab, cube)
    c.face(1, 0, 1, 0)
    c.points(0.01, corners(0.1, 0.1, 0.1, 0.09))


def case_cube_on_cube(backend):
    below, above = box(0, 0, 0, CUBE, IDENTITY), box(0, 0.19, 0, CUBE, IDENTITY)
    c = Contact(collide_backend(backend, 0, below, above), below, above)
    c.face(1, 0, 1, 0)
    c.points(0.01, corners(0.1, 0.1, 0.1, 0.09))


def case_turned_cube(backend):
    slab, cube = box(0, 0, 0, SLAB, IDENTITY), box(0, 0.19, 0, CUBE, axis_angle(0, 1, 0, math.pi / 4))
    c = Contact(collide_backend(backend, 0, slab, cube), slab, cube)
    c.face(1, 0, 1, 0)
    d = 0.1 * R2
    c.points(0.01, [[d, 0.09, 0], [-d, 0.09, 0], [0, 0.09, d], [0, 0.09, -d]])


def case_cube_over_edge(backend):
    slab, cube = box(0, 0, 0, SLAB, IDENTITY), box(0.25, 0.19, 0, CUBE, IDENTITY)
    c = Contact(collide_backend(backend, 0, slab, cube), slab, cube)
    c.face(1, 0, 1, 0)
    c.points(0.01, [[0.15, 0.09, 0.1], [0.15, 0.09, -0.1], [0.3, 0.09, 0.1], [0.3, 0.09, -0.1]])


def case_turned_cube_over_edge(backend):
    slab, cube = box(0, 0, 0, SLAB, IDENTITY), box(0.3, 0.19, 0, CUBE, axis_angle(0, 1, 0, math.pi / 4))
    c = Contact(collide_backend(backend, 0, slab, cube), slab, cube)
    c.face(1, 0, 1, 0)
    d = 0.1 * R2
    c.points(0.01, [[0.3 - d, 0.09, 0], [0.3, 0.09, d], [0.3, 0.09, -d]])


def case_other_way_round(backend):
    slab, cube = box(0, 0, 0, SLAB, IDENTITY), box(0, 0.19, 0, CUBE, IDENTITY)
    c = Contact(collide_backend(backend, 0, cube, slab), cube, slab)
    c.face(1, 0, -1, 0)
    c.points_on(0.01, corners(0.1, 0.1, 0.1, 0.09), corners(0.1, 0.1, 0.1, 0.1))


def case_crossed_edges(backend):
    top = 0.1 * R2
    below = box(0, 0, 0, CUBE, axis_angle(0, 0, 1, math.pi / 4))
    above = box(0, 2 * top - 0.01, 0, CUBE, axis_angle(1, 0, 0, math.pi / 4))
    m = collide_backend(backend, 0, below, above)
    c = Contact(m, below, above)
    assert m[B.AXIS] == 6 + 3 * 2
    c.normal(0, 1, 0)
    c.points_on(0.01, [[0, top, 0]], [[0, top - 0.01, 0]])


def case_corner_into_face(backend):
    tilt = math.acos(1 / math.sqrt(3))
    reach = 0.1 * math.sqrt(3)
    slab = box(0, 0, 0, SLAB, IDENTITY)
    cube = box(0, 0.1 + reach - 0.01, 0, CUBE, axis_angle(-1, 0, 1, tilt))
    c = Contact(collide_backend(backend, 0, slab, cube), slab, cube)
    c.face(1, 0, 1, 0)
    c.points_on(0.01, [[0, 0.1, 0]], [[0, 0.09, 0]])


def case_axis_of_second_parts(backend):
    m = collide_backend(backend, 0, box(0, 0, 0, CUBE, IDENTITY),
                        box(0.24, 0.24, 0, CUBE, axis_angle(0, 0, 1, math.pi / 4)))
    assert m[B.COUNT] == 0


def case_margin(backend):
    slab, cube = box(0, 0, 0, SLAB, IDENTITY), box(0, 0.205, 0, CUBE, IDENTITY)
    assert collide_backend(backend, 0, slab, cube)[B.COUNT] == 0
    c = Contact(collide_backend(backend, 0.01, slab, cube), slab, cube)
    c.face(1, 0, 1, 0)
    c.points(-0.005, corners(0.1, 0.1, 0.1, 0.105))


def case_ball_on_slab(backend):
    slab, b = box(0, 0, 0, SLAB, IDENTITY), ball(0, 0.14, 0, 0.05)
    c = Contact(collide_backend(backend, 0, slab, b), slab, b)
    c.face(B.SPHERE_BOX, 0, 1, 0)
    c.points_on(0.01, [[0, 0.1, 0]], [[0, 0.09, 0]])


def case_ball_first(backend):
    slab, b = box(0, 0, 0, SLAB, IDENTITY), ball(0, 0.14, 0, 0.05)
    c = Contact(collide_backend(backend, 0, b, slab), b, slab)
    c.face(B.SPHERE_BOX, 0, -1, 0)
    c.points_on(0.01, [[0, 0.09, 0]], [[0, 0.1, 0]])


def case_ball_over_edge(backend):
    slab, b = box(0, 0, 0, SLAB, IDENTITY), ball(0.33, 0.13, 0, 0.05)
    c = Contact(collide_backend(backend, 0, slab, b), slab, b)
    d = 1 / R2
    c.face(B.SPHERE_BOX, d, d, 0)
    depth = 0.05 - 0.03 * R2
    c.points_on(depth, [[0.3, 0.1, 0]], [[0.33 - 0.05 * d, 0.13 - 0.05 * d, 0]])


def case_ball_centre_inside(backend):
    slab, b = box(0, 0, 0, SLAB, IDENTITY), ball(0.1, 0.09, 0.05, 0.05)
    c = Contact(collide_backend(backend, 0, slab, b), slab, b)
    c.face(B.SPHERE_BOX, 0, 1, 0)
    c.points_on(0.06, [[0.1, 0.1, 0.05]], [[0.1, 0.04, 0.05]])


def case_two_balls(backend):
    first, second = ball(0, 0, 0, 0.05), ball(0.08, 0, 0, 0.04)
    c = Contact(collide_backend(backend, 0, first, second), first, second)
    c.face(B.SPHERE_SPHERE, 1, 0, 0)
    c.points_on(0.01, [[0.05, 0, 0]], [[0.04, 0, 0]])


def case_ball_apart(backend):
    m = collide_backend(backend, 0, box(0, 0, 0, SLAB, IDENTITY), ball(0, 0.2, 0, 0.05))
    assert m[B.COUNT] == 0


CASES = [case_boxes_apart, case_cube_on_slab, case_cube_on_cube, case_turned_cube, case_cube_over_edge,
         case_turned_cube_over_edge, case_other_way_round, case_crossed_edges, case_corner_into_face,
         case_axis_of_second_parts, case_margin, case_ball_on_slab, case_ball_first, case_ball_over_edge,
         case_ball_centre_inside, case_two_balls, case_ball_apart]


def random_pairs(pairs=500, seed=19):
    """BoxContactTest.everyPointLiesOnBothBoxesAtItsDepth's boxes, from java.util.Random(19)."""
    rnd = JavaRandom(seed)
    solids = []
    for k in range(2 * pairs):
        half = (0.03 + 0.12 * rnd.next_double(), 0.03 + 0.12 * rnd.next_double(), 0.03 + 0.12 * rnd.next_double())
        spread = 0 if k % 2 == 0 else 0.3
        cx = spread * (rnd.next_double() - 0.5)
        cy = spread * (rnd.next_double() - 0.5)
        cz = spread * (rnd.next_double() - 0.5)
        ax_ = rnd.next_double() - 0.5
        ay_ = rnd.next_double() - 0.5
        az_ = rnd.next_double() - 0.5
        ang = 4 * rnd.next_double()
        solids.append(box(cx, cy, cz, half, axis_angle(ax_, ay_, az_, ang)))
    return solids


def check_random_pairs(solids, allm):
    """The property checks of everyPointLiesOnBothBoxesAtItsDepth (BoxContactTest.java:191-254)."""
    pairs = len(solids) // 2
    touching = points = 0
    for p in range(pairs):
        m = allm[p * 40:(p + 1) * 40]
        first, second = solids[2 * p], solids[2 * p + 1]
        count = int(m[B.COUNT])
        assert count <= B.MOST_POINTS
        inner = min(first.half) + min(second.half)
        apart = math.hypot(math.hypot(second.centre[0] - first.centre[0], second.centre[1] - first.centre[1]),
                           second.centre[2] - first.centre[2])
        assert apart >= inner or count > 0, f"pair {p}: inner spheres overlap and no point"
        touching += count > 0
        points += count
        n = [float(m[B.NORMAL + a]) for a in range(3)]
        seen = []
        for k in range(count):
            at = B.POINTS + k * B.POINT_WORDS
            on_surface(m, at + B.ANCHOR_FIRST, first.half)
            on_surface(m, at + B.ANCHOR_SECOND, second.half)
            a = first.world(m, at + B.ANCHOR_FIRST)
            b = second.world(m, at + B.ANCHOR_SECOND)
            gap = (a[0] - b[0]) * n[0] + (a[1] - b[1]) * n[1] + (a[2] - b[2]) * n[2]
            assert abs(gap - float(m[at + B.DEPTH])) <= 1e-5, f"pair {p} point {k} depth"
            for j, s in enumerate(seen):
                assert math.hypot(math.hypot(b[0] - s[0], b[1] - s[1]), b[2] - s[2]) > 1e-6, f"pair {p}: {j}={k}"
            seen.append(b)
    assert touching > pairs // 2
    return touching, points


def on_surface(m, at, half):
    closest = float("inf")
    for a in range(3):
        inside = half[a] - abs(float(m[at + a]))
        assert inside > -1e-5
        closest = min(closest, inside)
    assert closest < 1e-5


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.__name__)
def test_oracle_hand_cases(case):
    case("oracle")


def test_oracle_random_pairs():
    solids = random_pairs()
    allm = collide_backend("oracle", 0, *solids)
    touching, points = check_random_pairs(solids, allm)
    assert touching > 250 and points > touching
