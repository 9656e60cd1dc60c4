"""A set of bodies put on a backend and stepped: the reference's test fixture BoxScene
(vexelray-sim-rigid-core/src/test/java/dev/vexelray/sim/rigid/box/BoxScene.java:17-262), restated.

Set the fields, then ``start(backend)``; ``advance`` steps, ``read`` brings the state back into the fields.
Backends: ``"oracle"`` (the CPU restatement under oracle/) and ``"gpu"`` (the CUDA library through its C-ABI).
"""
from __future__ import annotations

import numpy as np

from vxr import boxes as B


class BoxScene:
    def __init__(self, n: int):
        self.n = n
        f = lambda: np.zeros(n, dtype=np.float32)  # noqa: E731
        self.x, self.y, self.z = f(), f(), f()
        self.u, self.v, self.w = f(), f(), f()
        self.ax, self.ay, self.az = f(), f(), f()
        self.l = np.zeros((3, n), dtype=np.float32)
        self.q = np.zeros((4, n), dtype=np.float32)
        self.q[3] = 1
        self.half = np.zeros((3, n), dtype=np.float32)
        self.shape = f()
        self.im = np.ones(n, dtype=np.float32)
        self.gx, self.gy, self.gz = 0.0, -9.81, 0.0
        self.sx = self.sy = self.sz = 1.0
        self.dt = 1.0 / 60
        self.substeps = 10
        self.mu_static = 0.0
        self.mu_kinetic = 0.0
        self.mu_rolling = 0.0
        self.passes = B.WALL_PASSES
        self.margin = 0.005
        self.symmetric = False
        self.widest = None  # the half-diagonal the grid is sized by; None: from the halves, as BoxScene does
        self.cell = None  # a cell side to use in place of the reference rule's
        self.most_rounds = 0
        self.unplaced = 0
        self.unlisted = 0
        self.last = None
        self.world = None
        self.grid = None

    def sphere(self, s: int, r: float) -> "BoxScene":
        self.shape[s] = B.SPHERE_SHAPE
        self.half[:, s] = np.float32(r)
        return self

    def uniform(self, hx, hy, hz, mass) -> "BoxScene":
        self.half[0] = np.float32(hx)
        self.half[1] = np.float32(hy)
        self.half[2] = np.float32(hz)
        self.im[:] = np.float32(1 / mass)
        return self

    def param_bits(self):
        return B.params(self.dt / self.substeps, self.gx, self.gy, self.gz, self.sx, self.sy, self.sz,
                        self.mu_static, self.mu_kinetic, self.margin, self.mu_rolling)

    def _moment(self, s):
        return B.inertia(float(self.shape[s]), 1 / float(self.im[s]), float(self.half[0, s]), float(self.half[1, s]),
                         float(self.half[2, s]))

    def start(self, backend: str, **kw) -> "BoxScene":
        widest = self.widest if self.widest is not None else B.widest_half_diagonal(self.half)
        self.grid = B.grid(self.sx, self.sy, self.sz, widest, self.margin) if self.n > 1 else None
        if self.cell is not None and self.grid is not None:
            self.grid = B.covering(self.sx, self.sy, self.sz, self.cell)
        for s in range(self.n):
            if self.im[s] <= 0:
                continue
            spun = B.momentum([float(self.ax[s]), float(self.ay[s]), float(self.az[s])],
                              [float(c) for c in self.q[:, s]], self._moment(s))
            self.l[:, s] = np.float32(spun)
        if backend == "oracle":
            from oracle.box import OracleBoxWorld
            self.world = OracleBoxWorld(self.n, self.substeps, self.passes, self.symmetric, self.grid,
                                        threads=kw.get("threads", False))
            for name, vals in (("x", self.x), ("y", self.y), ("z", self.z), ("u", self.u), ("v", self.v),
                               ("w", self.w), ("lx", self.l[0]), ("ly", self.l[1]), ("lz", self.l[2]),
                               ("qx", self.q[0]), ("qy", self.q[1]), ("qz", self.q[2]), ("qw", self.q[3]),
                               ("im", self.im), ("hx", self.half[0]), ("hy", self.half[1]), ("hz", self.half[2]),
                               ("shape", self.shape)):
                self.world.set_field(name, vals)
            self.world.set_params(self.param_bits())
        elif backend == "gpu":
            from vxr.box_simulation import BoxSimulation
            self.world = BoxSimulation(self.n, self.substeps, self.passes, self.symmetric, self.grid, **kw)
            self.world.start_momentum(self.x, self.y, self.z, self.u, self.v, self.w, self.l, self.q, self.half,
                                      self.shape, self.im, self.param_bits())
        else:
            raise ValueError(backend)
        return self

    def advance(self, frames: int) -> "BoxScene":
        for _ in range(frames):
            self.last = self.world.step(1)
            touching, points, rounds, unplaced, unlisted = self.last
            self.most_rounds = max(self.most_rounds, rounds)
            self.unplaced += unplaced
            self.unlisted += unlisted
        return self

    def advance_seconds(self, seconds: float) -> "BoxScene":
        return self.advance(int(round(seconds / self.dt)))

    def read(self) -> "BoxScene":
        names = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]
        into = [self.x, self.y, self.z, self.u, self.v, self.w, self.l[0], self.l[1], self.l[2], self.q[0],
                self.q[1], self.q[2], self.q[3]]
        for name, dst in zip(names, into):
            dst[:] = self.world.field(name)
        for s in range(self.n):
            if self.im[s] > 0:
                om = B.spin([float(c) for c in self.l[:, s]], [float(c) for c in self.q[:, s]], self._moment(s))
            else:
                om = [0.0, 0.0, 0.0]
            self.ax[s], self.ay[s], self.az[s] = om
        return self

    def diagnostics(self) -> B.Diagnostics:
        self.read()
        return B.diagnostics(self.x, self.y, self.z, self.u, self.v, self.w, self.l, self.q, self.half, self.shape,
                             self.im)

    def own_spin(self, s: int):
        turn = [float(c) for c in self.q[:, s]]
        return B.rotate(B.conjugate(turn), [float(self.ax[s]), float(self.ay[s]), float(self.az[s])])

    def deepest(self) -> float:
        """The deepest point of any manifold of the last step."""
        best = 0.0
        for m in self.world.touching_manifolds():
            cnt = int(m[B.COUNT])
            for c in range(cnt):
                best = max(best, float(m[B.POINTS + c * B.POINT_WORDS + B.DEPTH]))
        return best

    def close(self):
        if self.world is not None:
            self.world.close()
            self.world = None
