"""Spheres in a box put on a backend and stepped: the reference's sphere test fixture Scene
(vexelray-sim-rigid-core/src/test/java/dev/vexelray/sim/rigid/sphere/Scene.java:14-233), restated.

Set the fields, then ``start(backend)``; ``advance`` steps, ``read`` brings the state back into the fields.
Backends: ``"oracle"`` (the CPU restatement under oracle/) and ``"gpu"`` (the CUDA library through its C-ABI).
"""
from __future__ import annotations

import numpy as np

from vxr import spheres as S


class SphereScene:
    def __init__(self, n: int):
        self.n = n
        f = lambda: np.zeros(n, dtype=np.float32)  # noqa: E731
        self.x, self.y, self.z = f(), f(), f()
        self.u, self.v, self.w = f(), f(), f()
        self.ax, self.ay, self.az = f(), f(), f()
        self.r = f()
        self.im = np.ones(n, dtype=np.float32)
        self.gx, self.gy, self.gz = 0.0, -9.81, 0.0
        self.sx = self.sy = self.sz = 1.0
        self.dt = 1.0 / 60
        self.substeps = 10
        self.iterations = 1
        self.omega = 1.0
        self.averaged = True
        self.restitution = 0.0
        self.mu_static = 0.0
        self.mu_kinetic = 0.0
        self.mu_rolling = 0.0
        self.grid = False
        self.solve = S.JACOBI
        self.rounds = S.ROUNDS
        self.fixed_rounds = False
        self.waits = 0
        self.rounds_run = 0
        self.most_rounds = 0
        self.unlisted = 0
        self.world = None
        self.backend = None
        self.last = None

    def uniform(self, radius, mass) -> "SphereScene":
        self.r[:] = np.float32(radius)
        self.im[:] = np.float32(1 / mass)
        return self

    def widest(self) -> float:
        return float(np.max(2.0 * self.r.astype(np.float64))) if self.n else 0.0

    def param_bits(self):
        return S.params(self.dt / self.substeps, self.gx, self.gy, self.gz, self.sx, self.sy, self.sz, self.omega,
                        self.averaged, self.restitution, self.mu_static, self.mu_kinetic, self.mu_rolling)

    def solve_kind(self) -> int:
        if self.solve == S.GAUSS_SEIDEL_BY_CONTACT and self.fixed_rounds:
            return S.FIXED_ROUNDS
        return self.solve

    def start(self, backend: str, **kwargs) -> "SphereScene":
        gridded = self.grid or self.solve != S.JACOBI
        grid = S.covering(self.sx, self.sy, self.sz, self.widest()) if gridded else None
        friction = self.mu_static + self.mu_kinetic + self.mu_rolling > 0
        fields = {"x": self.x, "y": self.y, "z": self.z, "u": self.u, "v": self.v, "w": self.w, "ax": self.ax,
                  "ay": self.ay, "az": self.az, "r": self.r, "im": self.im}
        self.backend = backend
        if backend == "oracle":
            from oracle.sphere import OracleSphereWorld
            self.world = OracleSphereWorld(self.n, self.substeps, self.iterations, self.solve_kind(), grid,
                                           rounds=self.rounds, **kwargs)
            for name, values in fields.items():
                self.world.set_field(name, values)
            self.world.set_params(self.param_bits(), friction)
        elif backend == "gpu":
            from vxr.sphere_simulation import SphereSimulation
            self.world = SphereSimulation(self.n, self.substeps, self.iterations, grid, self.solve_kind(),
                                          rounds=self.rounds, **kwargs)
            self.world.load_state(fields, self.param_bits())
            self.world.friction(friction)
        else:
            raise ValueError(backend)
        return self

    def advance(self, frames: int) -> "SphereScene":
        for _ in range(frames):
            report = self.world.step()
            self.last = report
            if self.solve_kind() == S.GAUSS_SEIDEL_BY_CONTACT:
                waits, rounds, most, unlisted = report
                self.waits += waits
                self.rounds_run += rounds
                self.most_rounds = max(self.most_rounds, most)
                self.unlisted += unlisted
        return self

    def advance_seconds(self, seconds: float) -> "SphereScene":
        return self.advance(int(round(seconds / self.dt)))

    def read(self) -> "SphereScene":
        for name in ("x", "y", "z", "u", "v", "w", "ax", "ay", "az"):
            getattr(self, name)[:] = self.world.field(name)
        return self

    def orientation(self, s: int):
        return [float(self.world.field(k)[s]) for k in ("qx", "qy", "qz", "qw")]

    def floats(self, name: str) -> np.ndarray:
        return self.world.field(name)

    def shown(self) -> np.ndarray:
        return self.world.shown()

    def contact_count(self):
        return self.world.counts() if self.solve != S.JACOBI else None

    def diagnostics(self) -> S.Diagnostics:
        self.read()
        return S.diagnostics(self.x, self.y, self.z, self.u, self.v, self.w, self.ax, self.ay, self.az, self.r,
                             self.im, self.gy, self.sx, self.sy, self.sz)

    def close(self):
        if self.world is not None:
            self.world.close()
            self.world = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
