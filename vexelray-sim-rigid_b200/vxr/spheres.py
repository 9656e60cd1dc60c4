"""Host-side helpers of the sphere package: parameters, the grid, and diagnostics.

Restates the reference's host code (core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/):
``Spheres.params``/``rubs`` (core/sphere/Spheres.java:141-235), ``SphereGrid`` (core/sphere/SphereGrid.java:11-36),
the step's constants (core/sphere/SphereStep.java:48-59) and ``SphereDiagnostics.of``
(core/sphere/SphereDiagnostics.java:34-83, host double precision).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PARAM_COUNT = 13
H, GX, GY, GZ, SX, SY, SZ, OMEGA, AVERAGED, RESTITUTION, MU_STATIC, MU_KINETIC, MU_ROLLING = range(13)
INERTIA = 0.4
LIST_MARGIN = np.float32(0.02)
MOST_LISTED_SPHERES = 46_340

# How a pass solves (SphereStep.Solve): Jacobi, or Gauss-Seidel over the contact list run until done. The third is
# the reference's fixed-rounds run of the latter (Scene.fixedRounds): `rounds` rounds a pass, no friction rounds.
JACOBI, GAUSS_SEIDEL_BY_CONTACT, FIXED_ROUNDS = 0, 1, 2
ROUNDS = 32
BATCH = 8
CYCLE = 48
CONTACTS_PER_SPHERE = 6

# The 24 per-sphere fields, in the reference's order (Spheres.SPHERE, core/sphere/Spheres.java:240-241).
FIELDS = ["x", "y", "z", "u", "v", "w", "r", "im", "cx", "cy", "cz", "dx", "dy", "dz", "ax", "ay", "az", "tx", "ty",
          "tz", "qx", "qy", "qz", "qw"]
FIELD = {name: k for k, name in enumerate(FIELDS)}

SHOWN_STRIDE = 40
PRESSED_BEFORE = 8
PRESSED_AFTER = 20
TURNED_BEFORE = 32
TURNED_AFTER = 36
PRESSING_WORDS = 12
FLATTENING, LEAN, TRACE, LEAN_LENGTH = 0, 6, 9, 10

IMPULSE_WORDS = 7
WALL_IMPULSE_WORDS = 21
LISTED, MISSED, LONGEST = 0, 1, 2


def _bits(value: float) -> int:
    return int(np.array([value], dtype=np.float32).view(np.int32)[0])


def params(h, gx, gy, gz, sx, sy, sz, omega, averaged, restitution=0.0, mu_static=0.0, mu_kinetic=0.0,
           mu_rolling=0.0) -> np.ndarray:
    """The 13 parameter words as float bits (Spheres.params, core/sphere/Spheres.java:212-228); ValueError where the
    reference throws IllegalArgumentException."""
    for mu in (mu_static, mu_kinetic, mu_rolling):
        if not (mu >= 0) or math.isinf(mu):
            raise ValueError(f"friction coefficients are finite and at least 0, got {mu_static}, {mu_kinetic} and "
                             f"{mu_rolling}")
    if not (restitution >= 0) or not (restitution <= 1):
        raise ValueError(f"restitution is in [0, 1], got {restitution}")
    if not (h > 0) or not (sx > 0) or not (sy > 0) or not (sz > 0) or not (omega > 0) or not (omega <= 1):
        raise ValueError(f"h > 0, a box of positive size and 0 < omega <= 1, got h {h}, box {sx} x {sy} x {sz}, "
                         f"omega {omega}")
    words = [h, gx, gy, gz, sx, sy, sz, omega, 1.0 if averaged else 0.0, restitution, mu_static, mu_kinetic,
             mu_rolling]
    return np.array([_bits(v) for v in words], dtype=np.int32)


def rubs(words) -> bool:
    """Whether the parameters ask for friction or rolling resistance (Spheres.rubs :231-235), in f32 as Java adds."""
    f = np.asarray(words, dtype=np.int32).view(np.float32)
    return bool(np.float32(np.float32(f[MU_STATIC] + f[MU_KINETIC]) + f[MU_ROLLING]) > 0)


@dataclass(frozen=True)
class SphereGrid:
    """nx x ny x nz cubic cells of side `cell` from the origin; cell (ix, iy, iz) is key ix + nx (iy + ny iz)."""
    nx: int
    ny: int
    nz: int
    cell: float

    def __post_init__(self):
        if self.nx < 1 or self.ny < 1 or self.nz < 1 or not (self.cell > 0):
            raise ValueError(f"a grid of at least one cell, of positive size, got {self.nx} x {self.ny} x {self.nz} "
                             f"of {self.cell}")

    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def covering(sx: float, sy: float, sz: float, widest: float) -> SphereGrid:
    """The grid over the box, its cells as wide as the widest sphere (SphereGrid.covering :21-26)."""
    if not (widest > 0):
        raise ValueError(f"the widest sphere must have a positive diameter, got {widest}")
    count = lambda extent: max(1, int(math.ceil(extent / widest)))  # noqa: E731
    return SphereGrid(count(sx), count(sy), count(sz), float(np.float32(widest)))


@dataclass
class Diagnostics:
    """SphereDiagnostics: overlaps as shares of the smaller radius, energies in joules, momenta, fastest speed."""
    max_overlap: float
    max_wall: float
    kinetic: float
    rotational: float
    potential: float
    momentum: tuple
    angular: tuple
    max_speed: float
    broken: bool


def diagnostics(x, y, z, u, v, w, ax, ay, az, r, im, gy, sx, sy, sz) -> Diagnostics:
    """SphereDiagnostics.of (core/sphere/SphereDiagnostics.java:34-83), host f64; the pair overlap over every pair."""
    d = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    x, y, z, u, v, w, ax, ay, az, r, im = map(d, (x, y, z, u, v, w, ax, ay, az, r, im))
    n = len(x)
    broken = not all(np.all(np.isfinite(a)) for a in (x, y, z, u, v, w, ax, ay, az))
    max_overlap = 0.0
    if n > 1:
        p = np.stack([x, y, z], axis=1)
        for a in range(n - 1):
            dist = np.sqrt(np.sum((p[a] - p[a + 1:]) ** 2, axis=1))
            overlap = (r[a] + r[a + 1:] - dist) / np.minimum(r[a], r[a + 1:])
            max_overlap = max(max_overlap, float(np.max(overlap)))
    max_wall = 0.0
    for at, extent in ((x, sx), (y, sy), (z, sz)):
        max_wall = max(max_wall, float(np.max((r - at) / r)), float(np.max((at + r - extent) / r)))
    speed2 = u * u + v * v + w * w
    max_speed = float(np.sqrt(np.max(speed2))) if n else 0.0
    free = im > 0
    m = np.where(free, 1.0 / np.where(free, im, 1.0), 0.0)
    inertia = INERTIA * m * r * r
    spin2 = ax * ax + ay * ay + az * az
    rotational = float(np.sum(np.where(free, 0.5 * inertia * spin2, 0.0)))
    kinetic = float(np.sum(np.where(free, 0.5 * m * speed2 + 0.5 * inertia * spin2, 0.0)))
    potential = float(np.sum(np.where(free, m * -gy * y, 0.0)))
    momentum = tuple(float(np.sum(m * c)) for c in (u, v, w))
    angular = (float(np.sum(m * (y * w - z * v) + inertia * ax)),
               float(np.sum(m * (z * u - x * w) + inertia * ay)),
               float(np.sum(m * (x * v - y * u) + inertia * az)))
    return Diagnostics(max(0.0, max_overlap), max(0.0, max_wall), kinetic, rotational, potential, momentum, angular,
                       max_speed, broken)


def shown_at_start(x, y, z, r) -> np.ndarray:
    """The picture's buffer at the start (SphereSimulation.start, gui/SphereSimulation.java:154-178): before and after
    both this state, the radius, and both orientations the identity."""
    n = len(x)
    shown = np.zeros((n, SHOWN_STRIDE), dtype=np.float32)
    shown[:, 0] = shown[:, 4] = x
    shown[:, 1] = shown[:, 5] = y
    shown[:, 2] = shown[:, 6] = z
    shown[:, 3] = r
    shown[:, TURNED_BEFORE + 3] = shown[:, TURNED_AFTER + 3] = 1
    return shown.reshape(-1)
