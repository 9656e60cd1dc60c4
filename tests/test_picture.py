"""The picture: the reference's sphere and box fragment shaders (gui/SphereShader.java, gui/BoxShader.java over
gui/Picture.java) as CUDA, against the oracle's restatement (oracle/picture_oracle.cpp) bit for bit.

The reference holds no rendered pictures (its ShaderTest only lowers the shaders to SPIR-V), so the oracle is pinned
here by what can be worked out by hand in doubles: the sky's gradient, the floor's checker, an unsquashed sphere
seen head-on with its octants, a box face with its edge band. Tolerance for those: 1e-5 on every channel (1e-4 for a
sphere-shaped box body, whose f32 quadratic cancels), away from the places where a pixel can fall either way (a
silhouette, a checker line, an octant's border)."""
import numpy as np
import pytest

from oracle import picture as OP
from vxr import picture as P

SKY_LOW = np.array([0.16, 0.17, 0.19])
SKY_HIGH = np.array([0.05, 0.06, 0.08])
FLOOR_A = np.array([0.30, 0.31, 0.33])
FLOOR_B = np.array([0.24, 0.25, 0.27])
BODY_A = np.array([0.90, 0.55, 0.22])
BODY_B = np.array([0.30, 0.62, 0.86])
LIGHT = np.array([0.35, 0.85, 0.4]) / np.linalg.norm([0.35, 0.85, 0.4])
TOL = 1e-5


def rays(eye, right, up, forward, aspect, w, h):
    """Every pixel's unit ray in doubles: Picture.Frame (gui/Picture.java:96-106)."""
    u = (np.arange(w) + 0.5) / w
    v = (np.arange(h) + 0.5) / h
    px = (u * 2 - 1) * aspect * 0.5
    py = (1 - v * 2) * 0.5
    d = (np.asarray(forward)[None, None, :] + np.asarray(right)[None, None, :] * px[None, :, None]
         + np.asarray(up)[None, None, :] * py[:, None, None])
    return d / np.linalg.norm(d, axis=2, keepdims=True)


def lit(d, n, hit, pale):
    """Picture.shade in doubles."""
    n = n / np.linalg.norm(n)
    diffuse = max(0.0, float(n @ LIGHT))
    h = LIGHT - d
    nh = max(0.0, float(n @ h) / np.linalg.norm(h))
    spec = 0.35 * nh ** 24
    g = hit * 0.618034
    tint = g - np.floor(g)
    colour = (BODY_A * (1 - tint) + BODY_B * tint) * (1 - pale) + pale
    return colour * (0.22 + 0.78 * diffuse) + spec


def test_sky_alone_is_the_gradient_by_height():
    eye, right, up, fwd = (0.5, 0.5, -3.0), (1, 0, 0), (0, 1, 0), (0, 0, 1)
    w, h = 24, 16
    cam = P.camera(eye, right, up, fwd, 1.5, 0.0, (1, 1, 1), 0.0)
    got = OP.picture(OP.SPHERES, np.zeros(0), P.push_words(cam, 0), w, h)
    d = rays(eye, right, up, fwd, 1.5, w, h)
    upness = np.clip(d[..., 1] * 0.5 + 0.5, 0, 1)[..., None]
    want = SKY_LOW * (1 - upness) + SKY_HIGH * upness
    sky = d[..., 1] >= -1e-4  # where the ray cannot meet the floor
    assert sky[: h // 2].all()
    np.testing.assert_allclose(got[sky], want[sky], atol=TOL)
    # below the horizon the floor is met outside the box (it runs from z = 0, the eye is at z = -3 looking at it
    # from outside): still sky, except where the ray lands inside the box's footprint
    t = -0.5 / np.where(d[..., 1] < -1e-4, d[..., 1], -1)
    fx, fz = 0.5 + t * d[..., 0], -3.0 + t * d[..., 2]
    near = lambda x: (np.abs(x) < 1e-3) | (np.abs(x - 1) < 1e-3)  # noqa: E731
    outside = (d[..., 1] < -1e-4) & ~((fx > 0) & (fx < 1) & (fz > 0) & (fz < 1)) & ~near(fx) & ~near(fz)
    assert outside.sum() > 100
    np.testing.assert_allclose(got[outside], want[outside], atol=TOL)


def test_floor_is_the_checker_inside_the_box():
    eye, fwd, right = (0.5, 1.0, 0.5), (0, -1, 0), (1, 0, 0)
    up = tuple(np.cross(fwd, right))
    w = h = 40
    cam = P.camera(eye, right, up, fwd, 1.0, 0.0, (1, 1, 1), 0.0)
    got = OP.picture(OP.BOXES, np.zeros(0), P.push_words(cam, 0), w, h)
    d = rays(eye, right, up, fwd, 1.0, w, h)
    t = 1.0 / -d[..., 1]
    fx, fz = 0.5 + t * d[..., 0], 0.5 + t * d[..., 2]
    cx, cz = fx / 0.05, fz / 0.05
    odd = (np.floor(cx) + np.floor(cz)) % 2
    want = FLOOR_A * (1 - odd[..., None]) + FLOOR_B * odd[..., None]
    clear = (np.abs(cx - np.round(cx)) > 1e-3) & (np.abs(cz - np.round(cz)) > 1e-3)
    assert clear.sum() > 0.8 * w * h
    np.testing.assert_allclose(got[clear], want[clear], atol=TOL)
    assert len(np.unique(odd[clear])) == 2


def sphere_shown(centre_before, centre_after, r, q_before=(0, 0, 0, 1), q_after=(0, 0, 0, 1), pressing=None):
    s = np.zeros(40, np.float32)
    s[0:3], s[3], s[4:7] = centre_before, r, centre_after
    if pressing is not None:
        s[8:20] = pressing
        s[20:32] = pressing
    s[32:36], s[36:40] = q_before, q_after
    return s


def test_an_unsquashed_sphere_head_on_with_its_octants():
    """A sphere halfway between its two centres, unpressed: every pixel that meets it well inside its silhouette is
    lit with the outward normal there, pale where x y z > 0 in its own frame."""
    c0, c1, r = np.array([0.4, 0.5, 0.5]), np.array([0.6, 0.5, 0.5]), 0.2
    s = sphere_shown(c0, c1, r)
    eye, right, up, fwd = (0.5, 0.5, -1.0), (1, 0, 0), (0, 1, 0), (0, 0, 1)
    w = h = 96
    cam = P.camera(eye, right, up, fwd, 1.0, 0.5, (1, 1, 1), 1.5)
    got = OP.picture(OP.SPHERES, s, P.push_words(cam, 1), w, h)
    d = rays(eye, right, up, fwd, 1.0, w, h)
    c = (c0 + c1) / 2
    o = np.array(eye) - c
    half = d @ o
    disc = half ** 2 - (o @ o - r * r)
    checked = 0
    for j in range(h):
        for i in range(w):
            if disc[j, i] < 1e-3:
                assert disc[j, i] > 0 or np.allclose(got[j, i], got[j, i].clip(0, 1))
                continue
            t = -half[j, i] - np.sqrt(disc[j, i])
            p = o + t * d[j, i]
            if min(abs(p[0]), abs(p[1]), abs(p[2])) < 2e-3:
                continue  # an octant's border
            pale = 0.45 if p[0] * p[1] * p[2] > 0 else 0.0
            np.testing.assert_allclose(got[j, i], lit(d[j, i], p, 0.0, pale), atol=TOL)
            checked += 1
    assert checked > 300


def test_a_box_face_with_its_edge_band():
    """An axis-aligned box seen square on: its near face lit with the face's normal, the band along its edges dark
    by EDGE_LIGHT; and a sphere-shaped body beside it drawn as a sphere, in octants of its own frame."""
    body = np.zeros(40, np.float32)
    body[0:3] = body[4:7] = (0.5, 0.5, 0.5)
    body[8:11] = (0.2, 0.15, 0.1)
    body[12:16] = body[16:20] = (0, 0, 0, 1)
    ball = np.array([0.85, 0.5, 0.5])
    body[20:23] = body[24:27] = ball
    body[23] = 1.0  # the sphere shape
    body[28:31] = 0.08
    body[32:36] = body[36:40] = (0, 0, 0, 1)
    eye, right, up, fwd = (0.5, 0.5, -1.0), (1, 0, 0), (0, 1, 0), (0, 0, 1)
    w, h = 128, 128
    cam = P.camera(eye, right, up, fwd, 1.0, 0.0, (1, 1, 1), 0.0)
    got = OP.picture(OP.BOXES, body, P.push_words(cam, 2), w, h)
    d = rays(eye, right, up, fwd, 1.0, w, h)
    n = np.array([0.0, 0.0, -1.0])
    band = 0.06 * 0.1
    seen = edged = round_ = 0
    for j in range(h):
        for i in range(w):
            t = (0.4 - eye[2]) / d[j, i, 2]
            p = np.array(eye) + t * d[j, i] - 0.5
            gx, gy = 0.2 - abs(p[0]), 0.15 - abs(p[1])
            if min(gx, gy) > 1e-4 and abs(min(gx, gy) - band) > 1e-4:
                want = lit(d[j, i], n, 0.0, 0.0)
                if min(gx, gy) < band:
                    want = want * 0.55
                    edged += 1
                np.testing.assert_allclose(got[j, i], want, atol=TOL)
                seen += 1
            o = np.array(eye) - ball
            half = d[j, i] @ o
            disc = half ** 2 - (o @ o - 0.08 ** 2)
            if disc > 1e-4:
                q = o + (-half - np.sqrt(disc)) * d[j, i]
                if min(abs(q)) > 2e-3:
                    pale = 0.45 if q[0] * q[1] * q[2] > 0 else 0.0
                    # the quadratic in f32 loses |o|^2 / r^2 ~ 350 times its rounding to cancellation
                    np.testing.assert_allclose(got[j, i], lit(d[j, i], q, 1.0, pale), atol=1e-4)
                    round_ += 1
    assert seen > 500 and edged > 20 and round_ > 100


def test_bodies_nearer_hide_those_behind():
    """Two spheres on one line of sight: the nearer one is the one painted (its index sets its colour)."""
    a = sphere_shown((0.5, 0.5, 0.3), (0.5, 0.5, 0.3), 0.1)
    b = sphere_shown((0.5, 0.5, 0.7), (0.5, 0.5, 0.7), 0.15)
    eye, right, up, fwd = (0.5, 0.5, -1.0), (1, 0, 0), (0, 1, 0), (0, 0, 1)
    cam = P.camera(eye, right, up, fwd, 1.0, 0.0, (1, 1, 1), 0.0)
    front = OP.picture(OP.SPHERES, np.concatenate([a, b]), P.push_words(cam, 2), 9, 9)[4, 4]
    back = OP.picture(OP.SPHERES, np.concatenate([b, a]), P.push_words(cam, 2), 9, 9)[4, 4]
    d = np.array([0.0, 0.0, 1.0])
    np.testing.assert_allclose(front, lit(d, -d, 0.0, 0.0), atol=TOL)
    np.testing.assert_allclose(back, lit(d, -d, 1.0, 0.0), atol=TOL)


def test_orbit_camera_is_the_views():
    """RigidView.show's camera (gui/RigidView.java:63-73): the eye on the orbit about the box's centre, forward to
    the centre, right level, up = forward x right."""
    cam = P.orbit_camera((2.0, 1.0, 1.0), (0.0, 0.5, -2.0))
    assert np.allclose(cam.eye[:], (1.0, 1.0, -1.5))
    f = np.array(cam.forward[:])
    r = np.array(cam.right[:])
    u = np.array(cam.up[:])
    assert np.allclose(f, -np.array([0.0, 0.5, -2.0]) / np.linalg.norm([0.0, 0.5, -2.0]), atol=1e-6)
    assert abs(r[1]) < 1e-7 and abs(r @ f) < 1e-6 and abs(np.linalg.norm(r) - 1) < 1e-6
    assert np.allclose(u, np.cross(f, r), atol=1e-6) and u[1] > 0


# ---- on the GPU: the CUDA kernels against the oracle, bit for bit ------------------------------------------------


def sphere_pile_shown(steps=30):
    import sphere_cases as SC
    s = SC.until_done_pile()
    s.mu_static = s.mu_kinetic = 0.5
    s.start("gpu").advance(steps)
    shown = s.world.shown()
    extent = (s.sx, s.sy, s.sz)
    n = s.n
    s.close()
    return shown, n, extent


def box_pile_shown(steps=40):
    import box_cases as C
    sc = C.mixed_pile_scene()
    sc.start("gpu")
    sc.world.step_and_wait(steps)
    shown = sc.world.read_shown()
    extent = (sc.sx, sc.sy, sc.sz)
    n = sc.n
    sc.close()
    return shown, n, extent


def gpu_picture(shape, shown, n, cam, w, h):
    import torch
    s = torch.from_numpy(np.ascontiguousarray(shown, np.float32)).cuda()
    out = torch.full((h, w, 3), float("nan"), device="cuda")
    P.draw(shape, s, n, cam, w, h, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("squash", [0.0, 1.5, 4.0])
@pytest.mark.parametrize("alpha", [0.0, 0.37, 1.0])
def test_gpu_spheres_match_the_oracle(squash, alpha):
    shown, n, extent = sphere_pile_shown()
    assert np.abs(shown.reshape(n, 40)[:, 8:20]).max() > 0, "the pile presses"
    cam = P.orbit_camera(extent, (1.2, 0.9, -1.6), alpha=alpha, squash=squash, aspect=96 / 64)
    got = gpu_picture(P.SPHERES, shown, n, cam, 96, 64)
    want = OP.picture(OP.SPHERES, shown, P.push_words(cam, n), 96, 64)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("alpha", [0.0, 0.5, 1.0])
def test_gpu_boxes_and_sphere_shapes_match_the_oracle(alpha):
    shown, n, extent = box_pile_shown()
    shape = shown.reshape(n, 20)[:, 3]
    assert (shape > 0.5).any() and (shape < 0.5).any()
    cam = P.orbit_camera(extent, (0.8, 0.6, -1.4), alpha=alpha, aspect=80 / 72)
    got = gpu_picture(P.BOXES, shown, n, cam, 80, 72)
    want = OP.picture(OP.BOXES, shown, P.push_words(cam, n), 80, 72)
    np.testing.assert_array_equal(got, want)
    hits = (np.abs(got - OP.picture(OP.BOXES, shown, P.push_words(cam, 0), 80, 72)) > 0).any(2)
    assert hits.mean() > 0.05, "the bodies are in view"


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(1, 1), (17, 13), (33, 7)])
def test_gpu_ragged_sizes_and_no_bodies(w, h):
    shown, n, extent = sphere_pile_shown(5)
    cam = P.orbit_camera(extent, (0.3, 1.5, -0.9), squash=1.5, aspect=w / h)
    for count in (0, n):
        got = gpu_picture(P.SPHERES, shown, count, cam, w, h)
        want = OP.picture(OP.SPHERES, shown, P.push_words(cam, count), w, h)
        np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_gpu_picture_from_a_ring_frame_and_from_host_memory():
    """The world's step kept in the ring and drawn from the reader's frame equals the picture drawn from the state
    read back to the host; the host entry point gives the same."""
    import torch

    import sphere_cases as SC
    from vxr.shown_ring import SPHERES, ShownRing
    s = SC.until_done_pile()
    s.start("gpu").advance(12)
    ring = ShownRing()
    ring.install(SPHERES, s.n, (s.sx, s.sy, s.sz))
    ring.keep(s.world, 12)
    frame = ring.take()
    cam = P.orbit_camera(frame.extent[:], (1.0, 1.0, -1.0), alpha=0.25, squash=1.5)
    out = torch.empty((40, 40, 3), device="cuda")
    P.draw_frame(frame, cam, 40, 40, out)
    torch.cuda.synchronize()
    shown = s.world.shown()
    want = OP.picture(OP.SPHERES, shown, P.push_words(cam, s.n), 40, 40)
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    np.testing.assert_array_equal(P.draw_host(P.SPHERES, shown, s.n, cam, 40, 40), want)
    ring.close()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("pose", [(1.2, 0.8, -1.6), (0.05, 0.1, 0.02), (-0.4, 0.05, 0.3)])
def test_gpu_many_bodies_from_outside_and_inside_the_pile(pose):
    """Thousands of bodies, the camera outside the pile and inside it (bodies beside, behind and around the eye): the
    tiles keep only the bodies their rays can meet, and the picture is still the oracle's loop over every body."""
    from vxr import scenes
    sc = scenes.large_mixed(4096, seed=4, volume=(24.0, 12.0, 24.0))
    from vxr import learned as Lm
    w = Lm.settled_world(sc, 60, 10)
    shown = w.read_shown()
    n = sc["bodies"]
    extent = sc["walls"]
    w.close()
    cam = P.orbit_camera(extent, pose, alpha=0.3, aspect=160 / 120)
    got = gpu_picture(P.BOXES, shown, n, cam, 160, 120)
    want = OP.picture(OP.BOXES, shown, P.push_words(cam, n), 160, 120)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_gpu_eye_inside_a_sphere_and_spheres_behind():
    """Spheres around the eye (one holding it), behind it and ahead of it, unpressed and pressed."""
    rng = np.random.default_rng(11)
    n = 600
    s = np.zeros((n, 40), np.float32)
    s[:, 0:3] = rng.uniform(-1.0, 2.0, (n, 3))
    s[:, 4:7] = s[:, 0:3] + rng.normal(0, 0.01, (n, 3))
    s[:, 3] = rng.uniform(0.02, 0.2, n)
    s[:, 8:20] = np.abs(rng.normal(0, 0.05, (n, 12)))
    s[:, 20:32] = s[:, 8:20]
    q = rng.normal(size=(n, 4))
    s[:, 32:36] = q / np.linalg.norm(q, axis=1, keepdims=True)
    s[:, 36:40] = s[:, 32:36]
    eye = np.array([0.5, 0.5, 0.5], np.float32)
    s[0, 0:3] = s[0, 4:7] = eye + 0.01
    s[0, 3] = 0.05
    cam = P.camera(eye, (1, 0, 0), (0, 1, 0), (0, 0, 1), 1.0, 0.5, (1, 1, 1), 1.5)
    got = gpu_picture(P.SPHERES, s.ravel(), n, cam, 96, 96)
    want = OP.picture(OP.SPHERES, s.ravel(), P.push_words(cam, n), 96, 96)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_gpu_a_super_tile_past_its_list_tests_every_body():
    """17,000 small spheres strung along the view's axis: the super-tiles at the picture's centre keep more bodies
    than their lists hold and fall back to every body, the others use their lists; the picture is the oracle's."""
    n = 17000
    rng = np.random.default_rng(5)
    s = np.zeros((n, 40), np.float32)
    z = 1.0 + 0.002 * np.arange(n)
    s[:, 0] = 0.5 + rng.uniform(-0.002, 0.002, n) * z
    s[:, 1] = 0.5 + rng.uniform(-0.002, 0.002, n) * z
    s[:, 2] = z
    s[:, 4:7] = s[:, 0:3]
    s[:, 3] = 0.003
    s[:, 32:36] = s[:, 36:40] = (0, 0, 0, 1)
    cam = P.camera((0.5, 0.5, 0.0), (1, 0, 0), (0, 1, 0), (0, 0, 1), 1.0, 0.0, (1, 1, 40), 0.0)
    got = gpu_picture(P.SPHERES, s.ravel(), n, cam, 192, 192)
    want = OP.picture(OP.SPHERES, s.ravel(), P.push_words(cam, n), 192, 192)
    np.testing.assert_array_equal(got, want)
    assert (np.abs(got - OP.picture(OP.SPHERES, s.ravel(), P.push_words(cam, 0), 192, 192)) > 0).any()
