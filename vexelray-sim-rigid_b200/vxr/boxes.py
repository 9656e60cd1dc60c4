"""Host-side helpers of the box/mixed-body step: parameters, inertia, diagnostics.

Mirrors the reference's host code (paths inside sibarum/vexelray-sim-rigid,
core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/):

* ``params`` / ``softness`` / ``inertia``      core/box/Boxes.java:179-268
* ``grid``                                      core/box/BoxBroad.java:66-68 with core/sphere/SphereGrid.java:21-35
* ``shown_at_start``                            core/box/Boxes.java:827-842
* ``diagnostics`` / ``spin`` / ``momentum``     core/box/BoxDiagnostics.java:18-66

Everything here is double precision on the host, rounded to f32 where the reference rounds, exactly as the
reference's Java does it (a Java ``double`` is an IEEE binary64, as a Python float is).
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass

import numpy as np

PARAM_COUNT = 18
H, GX, GY, GZ, SX, SY, SZ, MU_STATIC, MU_KINETIC, MARGIN = range(10)
BIAS, MASS_SCALE, IMPULSE_SCALE, STATIC_BIAS, STATIC_MASS_SCALE, STATIC_IMPULSE_SCALE = range(10, 16)
PUSH_SPEED, MU_ROLLING = 16, 17

CONTACT_HERTZ = 150.0
DAMPING_RATIO = 10.0
PUSH = 3.0
WALL_PASSES = 4
BOX_SHAPE = 0.0
SPHERE_SHAPE = 1.0
SPHERE_INERTIA = 0.4

SHOWN_STRIDE = 20
CENTRE_BEFORE, SHAPE, CENTRE_AFTER, HALF, TURNED_BEFORE, TURNED_AFTER = 0, 3, 4, 8, 12, 16

#: The most partners a body lists (BoxBroad.SLOTS) and the most rounds a step colours into (BoxStep.MOST_ROUNDS).
SLOTS = 32
MOST_ROUNDS = 32

#: Manifold layout (BoxContact.java:85-96) and impulse record (BoxPairs.java:48-50).
MANIFOLD_WORDS, NORMAL, COUNT, AXIS, POINTS, POINT_WORDS = 40, 0, 3, 4, 8, 8
ANCHOR_FIRST, ANCHOR_SECOND, DEPTH, MOST_POINTS = 0, 3, 6, 4
IMPULSE_WORDS, POINT_IMPULSE = 28, 7
SPHERE_BOX, SPHERE_SPHERE = 15, 16


def f32bits(value: float) -> int:
    """``Float.floatToRawIntBits((float) value)`` as a signed 32-bit int."""
    return struct.unpack("<i", struct.pack("<f", value))[0]


def bits_f32(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<i", bits))[0]


def softness(hertz: float, zeta: float, h: float) -> list[float]:
    """Box2D's ``b2MakeSoft``: ``[bias rate, mass scale, impulse scale]`` (Boxes.java:242-251)."""
    if hertz == 0:
        return [0.0, 1.0, 0.0]
    omega = 2 * math.pi * hertz
    a1 = 2 * zeta + h * omega
    a2 = h * omega * a1
    a3 = 1 / (1 + a2)
    return [omega / a1, a2 * a3, a3]


def params(h, gx, gy, gz, sx, sy, sz, mu_static=0.0, mu_kinetic=0.0, margin=0.0, mu_rolling=0.0) -> list[int]:
    """The 18 parameter words (f32 bits as ints), Boxes.params (Boxes.java:212-234).

    Raises ``ValueError`` where the reference throws ``IllegalArgumentException``.
    """
    if not (mu_rolling >= 0) or math.isinf(mu_rolling):
        raise ValueError(f"rolling resistance is finite and at least 0, got {mu_rolling}")
    if not (margin >= 0) or math.isinf(margin):
        raise ValueError(f"a margin is finite and at least 0, got {margin}")
    if not (h > 0) or not (sx > 0) or not (sy > 0) or not (sz > 0):
        raise ValueError(f"h > 0 and a box of positive size, got h {h}, box {sx} x {sy} x {sz}")
    if not (mu_static >= 0) or not (mu_kinetic >= 0) or math.isinf(mu_static) or math.isinf(mu_kinetic):
        raise ValueError(f"friction finite and at least 0, got {mu_static} and {mu_kinetic}")
    hertz = min(CONTACT_HERTZ, 0.25 / h)
    soft = softness(hertz, DAMPING_RATIO, h)
    stiff = softness(2 * hertz, DAMPING_RATIO, h)
    values = [h, gx, gy, gz, sx, sy, sz, mu_static, mu_kinetic, margin, soft[0], soft[1], soft[2], stiff[0],
              stiff[1], stiff[2], PUSH, mu_rolling]
    return [f32bits(v) for v in values]


def inertia(shape: float, m: float, hx: float, hy: float, hz: float) -> list[float]:
    """Principal moments by shape (Boxes.java:257-268): a box's ``m (b² + c²) / 3``, a sphere's ``⅖ m r²``."""
    if shape > 0.5:
        moment = SPHERE_INERTIA * m * hx * hx
        return [moment, moment, moment]
    return [m * (hy * hy + hz * hz) / 3, m * (hx * hx + hz * hz) / 3, m * (hx * hx + hy * hy) / 3]


@dataclass(frozen=True)
class Grid:
    """The broad phase's grid (SphereGrid.java:11-36): ``nx × ny × nz`` cubic cells of side ``cell``."""
    nx: int
    ny: int
    nz: int
    cell: float  # an f32 value

    def __post_init__(self):
        if self.nx < 1 or self.ny < 1 or self.nz < 1 or not (self.cell > 0):
            raise ValueError(f"a grid of at least one cell, of positive size, got {self.nx} x {self.ny} x "
                             f"{self.nz} of {self.cell}")

    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def covering(sx: float, sy: float, sz: float, widest: float) -> Grid:
    """SphereGrid.covering (SphereGrid.java:21-35)."""
    if not (widest > 0):
        raise ValueError(f"the widest sphere must have a positive diameter, got {widest}")

    def cells(extent):
        return max(1, int(math.ceil(extent / widest)))

    return Grid(cells(sx), cells(sy), cells(sz), float(np.float32(widest)))


def grid(sx: float, sy: float, sz: float, widest_half_diagonal: float, margin: float) -> Grid:
    """BoxBroad.grid (BoxBroad.java:66-68): cells as wide as the widest bounding sphere plus the margin."""
    return covering(sx, sy, sz, 2 * widest_half_diagonal + margin)


def widest_half_diagonal(half: np.ndarray) -> float:
    """The widest body's half-diagonal, as the reference's scene fixture sums it in f32 (BoxScene.java:121-125)."""
    h = np.asarray(half, dtype=np.float32)
    s = (h[0] * h[0] + h[1] * h[1]) + h[2] * h[2]
    return float(np.sqrt(np.max(s).astype(np.float64))) if h.shape[1] else 0.0


def shown_at_start(x, y, z, q, half, shape) -> np.ndarray:
    """``shown`` from the starting state, before and after both the start (Boxes.java:827-842)."""
    n = len(x)
    shown = np.zeros((n, SHOWN_STRIDE), dtype=np.float32)
    for a, c in enumerate((x, y, z)):
        shown[:, CENTRE_BEFORE + a] = c
        shown[:, CENTRE_AFTER + a] = c
        shown[:, HALF + a] = half[a]
    shown[:, SHAPE] = shape
    for k in range(4):
        shown[:, TURNED_BEFORE + k] = q[k]
        shown[:, TURNED_AFTER + k] = q[k]
    return shown.reshape(-1)


# --- diagnostics, in doubles (BoxDiagnostics.java) --------------------------------------------------------------

def rotate(q, p):
    """``p`` turned by the unit quaternion ``q`` (x, y, z, w), BoxDiagnostics.rotate :46-53."""
    ax = (q[0], q[1], q[2])
    t = _cross(ax, p)
    t = [2 * t[0], 2 * t[1], 2 * t[2]]
    qt = _cross(ax, t)
    return [p[0] + q[3] * t[0] + qt[0], p[1] + q[3] * t[1] + qt[1], p[2] + q[3] * t[2] + qt[2]]


def conjugate(q):
    return [-q[0], -q[1], -q[2], q[3]]


def spin(l, q, moment):
    """Angular velocity in the world's frame from angular momentum ``l`` (BoxDiagnostics.spin)."""
    own = rotate(conjugate(q), l)
    return rotate(q, [own[0] / moment[0], own[1] / moment[1], own[2] / moment[2]])


def momentum(omega, q, moment):
    """Angular momentum in the world's frame of a body spinning at ``omega`` (BoxDiagnostics.momentum)."""
    own = rotate(conjugate(q), omega)
    return rotate(q, [own[0] * moment[0], own[1] * moment[1], own[2] * moment[2]])


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


@dataclass
class Diagnostics:
    kinetic: float
    rotational: float
    momentum: list
    angular: list


def diagnostics(x, y, z, u, v, w, l, q, half, shape, im) -> Diagnostics:
    """BoxDiagnostics.of (BoxDiagnostics.java:18-43): moving energy, momentum and angular momentum, in doubles.

    Vectorised with numpy in float64; the sums run in the same per-body order as the reference's loop only up
    to numpy's pairwise summation, which is a double-precision diagnostic either way.
    """
    im = np.asarray(im, dtype=np.float32)
    live = im > 0
    m = 1.0 / im[live].astype(np.float64)
    at = np.stack([np.asarray(c, np.float32)[live].astype(np.float64) for c in (x, y, z)])
    vel = np.stack([np.asarray(c, np.float32)[live].astype(np.float64) for c in (u, v, w)])
    spun = np.stack([np.asarray(c, np.float32)[live].astype(np.float64) for c in l])
    qq = np.stack([np.asarray(c, np.float32)[live].astype(np.float64) for c in q])
    hh = np.stack([np.asarray(c, np.float32)[live].astype(np.float64) for c in half])
    sh = np.asarray(shape, np.float32)[live]
    sphere = sh > 0.5
    mom = np.empty_like(hh)
    mom[0] = np.where(sphere, SPHERE_INERTIA * m * hh[0] * hh[0], m * (hh[1] ** 2 + hh[2] ** 2) / 3)
    mom[1] = np.where(sphere, SPHERE_INERTIA * m * hh[0] * hh[0], m * (hh[0] ** 2 + hh[2] ** 2) / 3)
    mom[2] = np.where(sphere, SPHERE_INERTIA * m * hh[0] * hh[0], m * (hh[0] ** 2 + hh[1] ** 2) / 3)
    own = _vrotate(-qq[0], -qq[1], -qq[2], qq[3], spun)
    omega = _vrotate(qq[0], qq[1], qq[2], qq[3], own / mom)
    orbit = np.stack([at[1] * vel[2] - at[2] * vel[1], at[2] * vel[0] - at[0] * vel[2],
                      at[0] * vel[1] - at[1] * vel[0]])
    kinetic = float(np.sum(0.5 * m * vel * vel))
    rotational = float(np.sum(0.5 * spun * omega))
    mtm = [float(np.sum(m * vel[a])) for a in range(3)]
    ang = [float(np.sum(m * orbit[a] + spun[a])) for a in range(3)]
    return Diagnostics(kinetic + rotational, rotational, mtm, ang)


def _vrotate(qx, qy, qz, qw, p):
    t = np.stack([qy * p[2] - qz * p[1], qz * p[0] - qx * p[2], qx * p[1] - qy * p[0]]) * 2
    qt = np.stack([qy * t[2] - qz * t[1], qz * t[0] - qx * t[2], qx * t[1] - qy * t[0]])
    return p + qw * t + qt
