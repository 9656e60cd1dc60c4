"""Seeded synthetic scenes of the shapes the benchmark configurations name.

No public dataset is involved: each scene is drawn from numpy's PCG64 with a fixed seed, with the sizes and
distributions of its configuration. A scene is a dict of f32 arrays (x y z u v w lx ly lz qx qy qz qw im hx hy
hz shape) plus the walled box, step shape and parameters, ready for BoxSimulation.start_momentum (or the
oracle's world).
"""
from __future__ import annotations

import math

import numpy as np

from . import boxes as B

FIELDS = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw", "im", "hx", "hy", "hz", "shape"]


def _random_quaternions(rng, n):
    """Uniformly random unit quaternions (Shoemake's method)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    return np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3),
                     b * np.cos(2 * np.pi * u3)])


def large_mixed(bodies: int = 262_144, seed: int = 1, volume=(128.0, 64.0, 128.0), sphere_share: float = 0.8,
                mu: float = 0.5, mu_rolling: float = 0.1, margin: float = 0.005, dt: float = 1 / 120,
                substeps: int = 4, sweeps: int = 10, height: float | None = None) -> dict:
    """The large mixed scene: 80% spheres (radius log-uniform in 0.2-0.8 m), 20% boxes (half-extents uniform in
    0.2-0.6 m, uniformly random orientations), centres uniform in a 128 x 64 x 128 m volume above the floor,
    velocities N(0, 1 m/s) per axis, densities uniform in 500-2000 kg/m^3; dt 1/120 s, 4 substeps, 10 sweeps.

    The walls are the reference's walled box [0, sx] x [0, sy] x [0, sz] (core/box/Boxes.java:89-90): the volume's
    footprint, and a ceiling twice the volume's height. Friction and rolling resistance are not fixed by the
    configuration; mu 0.5 and mu_r 0.1 are used (the reference's own tests use 0.5 and 0.1-0.3).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    n = bodies
    vx, vy, vz = volume
    sphere = rng.random(n) < sphere_share
    radius = np.exp(rng.uniform(math.log(0.2), math.log(0.8), n))
    halves = rng.uniform(0.2, 0.6, (3, n))
    half = np.where(sphere, radius, halves)
    q = _random_quaternions(rng, n)
    q[:, sphere] = np.array([0.0, 0.0, 0.0, 1.0])[:, None]
    edge = 1.05  # no body starts in a wall: the widest reaches 1.04 m from its centre
    x = rng.uniform(edge, vx - edge, n)
    y = rng.uniform(edge, vy + edge, n)
    z = rng.uniform(edge, vz - edge, n)
    vel = rng.normal(0.0, 1.0, (3, n))
    density = rng.uniform(500.0, 2000.0, n)
    volume_of = np.where(sphere, 4.0 / 3.0 * np.pi * radius ** 3, 8.0 * halves[0] * halves[1] * halves[2])
    im = 1.0 / (density * volume_of)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    scene = {
        "x": f32(x), "y": f32(y), "z": f32(z), "u": f32(vel[0]), "v": f32(vel[1]), "w": f32(vel[2]),
        "lx": np.zeros(n, np.float32), "ly": np.zeros(n, np.float32), "lz": np.zeros(n, np.float32),
        "qx": f32(q[0]), "qy": f32(q[1]), "qz": f32(q[2]), "qw": f32(q[3]), "im": f32(im),
        "hx": f32(half[0]), "hy": f32(half[1]), "hz": f32(half[2]),
        "shape": np.where(sphere, B.SPHERE_SHAPE, B.BOX_SHAPE).astype(np.float32),
    }
    sy = height if height is not None else 2 * vy
    h3 = np.stack([scene["hx"], scene["hy"], scene["hz"]])
    # the widest bounding sphere (BoxBroad.grid's rule): a box's half-diagonal, a sphere's radius
    boxes_only = h3[:, ~sphere] if (~sphere).any() else np.zeros((3, 1), np.float32)
    widest = max(B.widest_half_diagonal(boxes_only), float(np.max(scene["hx"][sphere])) if sphere.any() else 0.0)
    scene.update({
        "bodies": n, "walls": (vx, sy, vz), "dt": dt, "substeps": substeps, "sweeps": sweeps, "margin": margin,
        "mu": mu, "mu_rolling": mu_rolling, "widest": widest,
        "grid": B.grid(vx, sy, vz, widest, margin),
        "params": B.params(dt / substeps, 0.0, -9.81, 0.0, vx, sy, vz, mu, mu, margin, mu_rolling),
        "name": f"large mixed scene, {n} bodies ({sphere_share:.0%} spheres), seed {seed}",
    })
    return scene


def sub_volume(bodies_full: int, fraction: float, seed: int = 1) -> dict:
    """The large mixed scene's distribution over a fraction of its volume (same body density): a bounded
    sample for a CPU baseline. The footprint shrinks, the height stays."""
    side = math.sqrt(fraction)
    return large_mixed(int(round(bodies_full * fraction)), seed=seed, volume=(128.0 * side, 64.0, 128.0 * side))


def towers(seed: int = 1, towers_x: int = 8, towers_z: int = 8, height: int = 64, spacing: float = 3.0,
           density: float = 1000.0, mu: float = 0.6, margin: float = 0.005, dt: float = 1 / 60, substeps: int = 8,
           sweeps: int = 16) -> dict:
    """Box stacking: 8 x 8 = 64 towers of 64 boxes on a ground grid at 3 m spacing (4,096 boxes). Half-extents
    seeded uniform in 0.25-0.75 m per axis; each box a seeded yaw in +-15 degrees and a seeded offset of +-0.02 m
    from its tower's axis; each box set down on the one below (its bottom face on the lower box's top). mu 0.6, no
    restitution, dt 1/60 s with 8 substeps and 16 sweeps; 1,000 steps, judged by penetration and energy drift.
    The configuration names no density: 1000 kg/m^3. The walls: the ground grid's footprint, and a ceiling above the
    tallest tower."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = towers_x * towers_z * height
    half = rng.uniform(0.25, 0.75, (3, n))
    yaw = np.radians(rng.uniform(-15.0, 15.0, n))
    off = rng.uniform(-0.02, 0.02, (2, n))
    x, y, z = np.zeros(n), np.zeros(n), np.zeros(n)
    k = 0
    for i in range(towers_x):
        for j in range(towers_z):
            top = 0.0
            for _ in range(height):
                x[k] = spacing * (i + 0.5) + off[0, k]
                z[k] = spacing * (j + 0.5) + off[1, k]
                y[k] = top + half[1, k]
                top = y[k] + half[1, k]
                k += 1
    sx, sz = spacing * towers_x, spacing * towers_z
    sy = float(np.max(y + half[1])) + 10.0
    q = np.stack([np.zeros(n), np.sin(yaw / 2), np.zeros(n), np.cos(yaw / 2)])
    im = 1.0 / (density * 8.0 * half[0] * half[1] * half[2])
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    zero = np.zeros(n, np.float32)
    scene = {"x": f32(x), "y": f32(y), "z": f32(z), "u": zero.copy(), "v": zero.copy(), "w": zero.copy(),
             "lx": zero.copy(), "ly": zero.copy(), "lz": zero.copy(), "qx": f32(q[0]), "qy": f32(q[1]),
             "qz": f32(q[2]), "qw": f32(q[3]), "im": f32(im), "hx": f32(half[0]), "hy": f32(half[1]),
             "hz": f32(half[2]), "shape": np.full(n, B.BOX_SHAPE, np.float32)}
    widest = B.widest_half_diagonal(np.stack([scene["hx"], scene["hy"], scene["hz"]]))
    scene.update({"bodies": n, "walls": (sx, sy, sz), "dt": dt, "substeps": substeps, "sweeps": sweeps,
                  "margin": margin, "mu": mu, "widest": widest, "grid": B.grid(sx, sy, sz, widest, margin),
                  "params": B.params(dt / substeps, 0.0, -9.81, 0.0, sx, sy, sz, mu, mu, margin, 0.0),
                  "name": f"{towers_x * towers_z} towers of {height} boxes, seed {seed}"})
    return scene


def batched(scenes: int = 512, seed: int = 1, smallest: int = 64, largest: int = 4096, sphere_share: float = 0.7,
            dt: float = 1 / 60, substeps: int = 4, sweeps: int = 10, margin: float = 0.005,
            mu_rolling: float = 0.1) -> dict:
    """Independent scenes for one batched world: each scene's body count log-uniform in 64-4096, a 70/30
    sphere/box mix with the large mixed scene's size, orientation, velocity and density distributions, its own
    gravity tilted by up to 5 degrees about a random horizontal axis, and its own mu in 0.3-0.8 (static = kinetic).
    dt 1/60 s, 4 substeps; the configuration names no sweep count, so the large mixed scene's 10 are used.

    Each scene drops at the large mixed scene's body density (0.25 a cubic metre) into its own walled box a x a x a
    with a = (8 N)^(1/3) (bodies start in the lower half). Returns the concatenated fields (scene after scene), each
    scene's count, grid and 18 parameter words."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = np.round(np.exp(rng.uniform(math.log(smallest), math.log(largest), scenes))).astype(np.int32)
    parts, grids, words, walls = [], [], [], []
    for k in range(scenes):
        n = int(counts[k])
        a = (8.0 * n) ** (1.0 / 3.0)
        sc = large_mixed(n, seed=int(rng.integers(1 << 31)), volume=(a, a / 2, a), sphere_share=sphere_share,
                         dt=dt, substeps=substeps, sweeps=sweeps, margin=margin, mu_rolling=mu_rolling, height=a)
        tilt = math.radians(rng.uniform(-5.0, 5.0))
        about = rng.uniform(0.0, 2.0 * math.pi)
        g = (9.81 * math.sin(tilt) * math.cos(about), -9.81 * math.cos(tilt), 9.81 * math.sin(tilt) * math.sin(about))
        mu = float(rng.uniform(0.3, 0.8))
        sx, sy, sz = sc["walls"]
        words.append(B.params(dt / substeps, g[0], g[1], g[2], sx, sy, sz, mu, mu, margin, mu_rolling))
        grids.append(sc["grid"])
        walls.append((sx, sy, sz))
        parts.append(sc)
    out = {name: np.concatenate([p[name] for p in parts]) for name in FIELDS}
    out.update({
        "scenes": scenes, "counts": counts, "bodies": int(counts.sum()), "grids": grids,
        "params": np.stack(words), "walls": walls, "dt": dt, "substeps": substeps, "sweeps": sweeps,
        "margin": margin, "parts": parts,
        "name": f"{scenes} batched scenes, {int(counts.sum())} bodies ({sphere_share:.0%} spheres), seed {seed}",
    })
    return out


def sphere_lattice(seed: int = 1, nx: int = 16, ny: int = 8, nz: int = 8, spacing: float = 1.2,
                   jitter: float = 0.05, radius: float = 0.5, density: float = 1000.0, box: float = 20.0,
                   height: float = 40.0) -> dict:
    """The plain sphere scene: 16 x 8 x 8 = 1,024 spheres of radius 0.5 m and density 1000 kg/m^3 on a lattice at
    1.2 m, each jittered by a seeded uniform +-0.05 m per axis, at rest, dropping into an open 20 x 20 m box of
    static planes (the reference's walled box with its lid far above: `height`). dt 1/60 s with 4 substeps and 8
    iterations of Gauss-Seidel over the contact list, mu 0.5, restitution 0.2, grid cells 1.0 m; 600 steps.

    Lattice columns run along x (16, centred in the box's width), layers along y from 1 m up, rows along z (8,
    centred in its depth)."""
    from . import spheres as S
    rng = np.random.Generator(np.random.PCG64(seed))
    n = nx * ny * nz
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x0 = (box - (nx - 1) * spacing) / 2
    z0 = (box - (nz - 1) * spacing) / 2
    x = x0 + spacing * i.reshape(-1) + rng.uniform(-jitter, jitter, n)
    y = 1.0 + spacing * j.reshape(-1) + rng.uniform(-jitter, jitter, n)
    z = z0 + spacing * k.reshape(-1) + rng.uniform(-jitter, jitter, n)
    mass = density * 4.0 / 3.0 * math.pi * radius ** 3
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    dt, substeps = 1 / 60, 4
    return {
        "x": f32(x), "y": f32(y), "z": f32(z), "u": np.zeros(n, np.float32), "v": np.zeros(n, np.float32),
        "w": np.zeros(n, np.float32), "r": np.full(n, radius, np.float32), "im": np.full(n, 1 / mass, np.float32),
        "spheres": n, "walls": (box, height, box), "dt": dt, "substeps": substeps, "iterations": 8,
        "grid": S.covering(box, height, box, 2 * radius),
        "params": S.params(dt / substeps, 0.0, -9.81, 0.0, box, height, box, 1.0, True, 0.2, 0.5, 0.5, 0.0),
        "steps": 600,
        "name": f"sphere lattice {nx}x{ny}x{nz} = {n} spheres, r {radius} m, seed {seed}",
    }


def fields(scene: dict) -> list:
    return [scene[k] for k in FIELDS]


def _java_doubles(seed: int):
    """java.util.Random(seed).nextDouble(), again and again: the Java SE API's documented 48-bit linear
    congruential generator, nextDouble = ((next(26) << 27) + next(27)) * 2^-53."""
    mult, mask = 0x5DEECE66D, (1 << 48) - 1
    state = (seed ^ mult) & mask

    def nxt(bits):
        nonlocal state
        state = (state * mult + 0xB) & mask
        return state >> (48 - bits)

    while True:
        yield ((nxt(26) << 27) + nxt(27)) * (1.0 / (1 << 53))


# The reference's sphere sweep's solver settings (core tests, sphere/SphereSweepTest.java:20-48, :74-91): the name,
# substeps, solve ("gs" Gauss-Seidel over the contact list run until done, "jacobi" on the grid), averaged, mu.
PILE_SOLVERS = {
    "until done mu=0.5": (10, "gs", False, 0.5),
    "until done": (10, "gs", False, 0.0),
    "grid averaged omega=1": (10, "jacobi", True, 0.0),
}


def sphere_pile(side: int = 16, seed: int = 7, solver: str = "until done mu=0.5") -> dict:
    """The reference's sphere pile (core tests, sphere/SphereSweepTest.java:118-144, the large pile at side 16):
    side^3 spheres of radius 3 cm and mass 0.1 kg dropped as a loose lattice into a box 0.08 + 0.06 side wide and
    deep and 0.5 + 0.07 side tall, column x and row z jittered by java.util.Random(seed) (x drawn before z), layers
    0.07 m apart from 0.3 m up; dt 1/60 s, one pass a substep, gravity -9.81, no restitution. `solver` is one of
    PILE_SOLVERS. The reference times it over 240 frames at 60 Hz, after 2."""
    from . import spheres as S
    substeps, kind, averaged, mu = PILE_SOLVERS[solver]
    solve = S.GAUSS_SEIDEL_BY_CONTACT if kind == "gs" else S.JACOBI
    n = side ** 3
    rnd = _java_doubles(seed)
    x, y, z = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32)
    k = 0
    for i in range(side):
        for j in range(side):
            for l_ in range(side):
                x[k] = np.float32(0.07 + 0.06 * i + 0.005 * next(rnd))
                y[k] = np.float32(0.3 + 0.07 * j)
                z[k] = np.float32(0.07 + 0.06 * l_ + 0.005 * next(rnd))
                k += 1
    sx = sz = 0.08 + 0.06 * side
    sy = 0.5 + 0.07 * side
    dt = 1 / 60
    r = np.full(n, np.float32(0.03), np.float32)
    return {"x": x, "y": y, "z": z, "u": np.zeros(n, np.float32), "v": np.zeros(n, np.float32),
            "w": np.zeros(n, np.float32), "r": r, "im": np.full(n, np.float32(1 / 0.1), np.float32),
            "spheres": n, "walls": (sx, sy, sz), "dt": dt, "substeps": substeps, "iterations": 1, "solve": solve,
            "friction": mu > 0, "grid": S.covering(sx, sy, sz, 0.06),
            "params": S.params(dt / substeps, 0.0, -9.81, 0.0, sx, sy, sz, 1.0, averaged, 0.0, mu, mu, 0.0),
            "frames": 240, "name": f"sphere pile {side}^3 = {n} spheres, r 3 cm, {solver}, seed {seed}"}
