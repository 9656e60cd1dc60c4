"""Diagnostics computed on the GPU, against the same quantities computed on the host in doubles from the state read
back (BoxDiagnostics.of and SphereDiagnostics.of restated in vxr/boxes.py and vxr/spheres.py); and the box-stacking
configuration judged over its run by penetration and energy drift."""
import numpy as np
import pytest

import sphere_cases as SC
from vxr import boxes as B
from vxr import learned as Lm
from vxr import scenes

pytestmark = pytest.mark.gpu


def rotate(q, p):
    """q (4, n) applied to p (3, n), in doubles."""
    qx, qy, qz, qw = q
    t = 2 * np.stack([qy * p[2] - qz * p[1], qz * p[0] - qx * p[2], qx * p[1] - qy * p[0]])
    return p + qw * t + np.stack([qy * t[2] - qz * t[1], qz * t[0] - qx * t[2], qx * t[1] - qy * t[0]])


def host_penetrations(w, sc):
    x, y, z, u, v, wv, lx, ly, lz, qx, qy, qz, qw = [a.astype(np.float64) for a in w.state()]
    at = np.stack([x, y, z])
    q = np.stack([qx, qy, qz, qw])
    half = np.stack([sc["hx"], sc["hy"], sc["hz"]]).astype(np.float64)
    sphere = sc["shape"] > 0.5
    a, b, c, m, _ = w.touching()
    deepest = 0.0
    for t in range(len(a)):
        n = m[t, 0:3].astype(np.float64)
        for i in range(c[t]):
            pt = m[t, B.POINTS + i * B.POINT_WORDS:]
            ra = half[0, a[t]] * n if sphere[a[t]] else rotate(q[:, a[t]:a[t] + 1], pt[0:3, None].astype(np.float64))[:, 0]
            rb = -half[0, b[t]] * n if sphere[b[t]] else rotate(q[:, b[t]:b[t] + 1], pt[3:6, None].astype(np.float64))[:, 0]
            gap = float(np.dot((at[:, b[t]] + rb) - (at[:, a[t]] + ra), n))
            deepest = max(deepest, -gap)
    # past a wall: a sphere's surface, a box's corners
    ext = np.array(sc["walls"], np.float64)[:, None]
    wall = float(np.max(np.where(sphere, np.maximum(half[0] - at, at + half[0] - ext).max(0), -np.inf)))
    for cidx in range(8):
        off = np.stack([np.where((cidx >> k) & 1, half[k], -half[k]) for k in range(3)])
        p = at + rotate(q, off)
        worst = np.maximum(-p, p - ext).max(0)
        wall = max(wall, float(np.max(np.where(sphere, -np.inf, worst))))
    return deepest, max(wall, 0.0)


def test_gpu_box_diagnostics_match_the_host():
    sc = scenes.large_mixed(4096, seed=2, volume=(24.0, 12.0, 24.0))
    w = Lm.settled_world(sc, 220, 16)
    d = w.gpu_diagnostics()
    st = w.state()
    host = B.diagnostics(*st[:6], st[6:9], st[9:13], [sc["hx"], sc["hy"], sc["hz"]], sc["shape"], sc["im"])
    rel = lambda a, b: abs(a - b) / max(abs(b), 1e-12)  # noqa: E731
    assert rel(d["kinetic"], host.kinetic) < 1e-6
    assert rel(d["rotational"], host.rotational) < 1e-6
    for k in range(3):
        assert abs(d["momentum"][k] - host.momentum[k]) < 1e-6 * max(1.0, abs(host.momentum[k]))
        assert abs(d["angular"][k] - host.angular[k]) < 1e-6 * max(1.0, abs(host.angular[k]))
    im = sc["im"].astype(np.float64)
    g = float(np.float32(9.81))  # the parameter word's value
    potential = float(np.sum(np.where(im > 0, g * st[1].astype(np.float64) / np.where(im > 0, im, 1), 0)))
    assert rel(d["potential"], potential) < 1e-9
    deepest, wall = host_penetrations(w, sc)
    assert abs(d["max_penetration"] - deepest) < 2e-6
    assert abs(d["max_wall_penetration"] - wall) < 2e-6
    assert not d["broken"]
    w.close()


def test_gpu_sphere_diagnostics_match_the_host():
    s = SC.until_done_pile()
    s.mu_static = s.mu_kinetic = 0.5
    s.start("gpu").advance(20)
    d = s.world.gpu_diagnostics()
    host = s.diagnostics()
    assert abs(d.max_overlap - host.max_overlap) < 1e-6 * max(1.0, host.max_overlap)
    assert abs(d.max_wall - host.max_wall) < 1e-6
    for k in ("kinetic", "rotational", "potential", "max_speed"):
        assert abs(getattr(d, k) - getattr(host, k)) <= 1e-7 * max(1.0, abs(getattr(host, k))), k
    for k in range(3):
        assert abs(d.momentum[k] - host.momentum[k]) <= 1e-7 * max(1.0, abs(host.momentum[k]))
        assert abs(d.angular[k] - host.angular[k]) <= 1e-7 * max(1.0, abs(host.angular[k]))
    assert d.broken == host.broken
    s.close()


def test_gpu_box_towers_stand_without_penetration_or_energy_gain():
    """A 2 x 2 block of the stacking configuration's towers, 16 boxes tall, 300 steps at its 8 substeps and 16
    sweeps: nothing breaks, no contact sinks deeper than 5 mm, no box reaches past a wall by more than a millimetre,
    and the energy never rises (contact only takes energy)."""
    sc = scenes.towers(seed=3, towers_x=2, towers_z=2, height=16)
    w = Lm.settled_world(sc, 0, 16)
    first = w.gpu_diagnostics()
    e0 = first["kinetic"] + first["potential"]
    worst = 0.0
    for _ in range(30):
        w.step_and_wait(10)
        d = w.gpu_diagnostics()
        assert not d["broken"]
        worst = max(worst, d["max_penetration"])
        assert d["max_wall_penetration"] < 1e-3
        assert d["kinetic"] + d["potential"] <= e0 * (1 + 1e-5)
    assert worst < 5e-3
    w.close()


def host_contact_errors(w, sc, h, margin):
    """Each contact point's complementarity error, in doubles from the state read back."""
    x, y, z, u, v, wv, lx, ly, lz, qx, qy, qz, qw = [a.astype(np.float64) for a in w.state()]
    at, vel, spun = np.stack([x, y, z]), np.stack([u, v, wv]), np.stack([lx, ly, lz])
    q = np.stack([qx, qy, qz, qw])
    half = np.stack([sc["hx"], sc["hy"], sc["hz"]]).astype(np.float64)
    sphere = sc["shape"] > 0.5
    m = 1.0 / sc["im"].astype(np.float64)
    moment = np.where(sphere, 0.4 * m * half[0] ** 2, 0.0)
    moments = np.stack([np.where(sphere, moment, m * (half[1] ** 2 + half[2] ** 2) / 3),
                        np.where(sphere, moment, m * (half[0] ** 2 + half[2] ** 2) / 3),
                        np.where(sphere, moment, m * (half[0] ** 2 + half[1] ** 2) / 3)])
    conj = q * np.array([-1, -1, -1, 1.0])[:, None]
    omega = rotate(q, rotate(conj, spun) / moments)
    a, b, c, mf, _ = w.touching()
    out = []
    for t in range(len(a)):
        n = mf[t, 0:3].astype(np.float64)
        for i in range(c[t]):
            pt = mf[t, B.POINTS + i * B.POINT_WORDS:]
            ra = half[0, a[t]] * n if sphere[a[t]] else rotate(q[:, a[t]:a[t] + 1], pt[0:3, None].astype(np.float64))[:, 0]
            rb = -half[0, b[t]] * n if sphere[b[t]] else rotate(q[:, b[t]:b[t] + 1], pt[3:6, None].astype(np.float64))[:, 0]
            gap = float(np.dot((at[:, b[t]] + rb) - (at[:, a[t]] + ra), n))
            va = vel[:, a[t]] + np.cross(omega[:, a[t]], ra)
            vb = vel[:, b[t]] + np.cross(omega[:, b[t]], rb)
            vn = float(np.dot(vb - va, n))
            closing = h * max(0.0, -(vn + max(gap, 0.0) / h)) if gap <= margin else 0.0
            out.append(max(closing, max(0.0, -gap)))
    return np.sort(np.array(out))


def test_gpu_contact_errors_match_the_host():
    """The step-end complementarity error of every contact point (vxr_box_contact_errors) against the same
    quantity in doubles from the state read back, as sorted sets (the GPU lists points in round order)."""
    sc = scenes.large_mixed(2048, seed=4, volume=(16.0, 8.0, 16.0))
    w = Lm.settled_world(sc, 90, 16)
    got = np.sort(w.contact_errors())
    h = B.bits_f32(sc["params"][B.H])
    margin = B.bits_f32(sc["params"][B.MARGIN])
    want = host_contact_errors(w, sc, h, margin)
    assert len(got) == len(want) and len(got) > 100
    np.testing.assert_allclose(got, want, atol=2e-6, rtol=1e-4)
    assert want.max() > 0.0
    w.close()
