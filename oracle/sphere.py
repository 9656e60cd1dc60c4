"""CPU ORACLE — test infrastructure only. ctypes binding of the C++ restatement in ``sphere_oracle.cpp``.

Used by tests/, ``__graft_entry__.smoke()`` (as the checker) and bench.py's CPU-baseline leg; never by the
product path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import box

FIELDS = ["x", "y", "z", "u", "v", "w", "r", "im", "cx", "cy", "cz", "dx", "dy", "dz", "ax", "ay", "az", "tx", "ty",
          "tz", "qx", "qy", "qz", "qw"]
SHOWN_STRIDE = 40
IMPULSE_WORDS = 7
WALL_IMPULSE_WORDS = 21

_bound: set = set()


def lib(threads: bool = False) -> ctypes.CDLL:
    L = box.lib(threads)
    if id(L) not in _bound:
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.orc_sphere_create.restype = vp
        L.orc_sphere_create.argtypes = [i, i, i, i, i, i, i, i, f, i]
        L.orc_sphere_destroy.argtypes = [vp]
        L.orc_sphere_set_field.argtypes = [vp, i, vp]
        L.orc_sphere_get_field.argtypes = [vp, i, vp]
        L.orc_sphere_set_params.argtypes = [vp, vp, i]
        L.orc_sphere_step.argtypes = [vp, i, vp]
        L.orc_sphere_step.restype = i
        L.orc_sphere_shown.argtypes = [vp, vp]
        L.orc_sphere_set_shown.argtypes = [vp, vp]
        L.orc_sphere_contacts.argtypes = [vp, vp, vp, i]
        L.orc_sphere_contacts.restype = i
        L.orc_sphere_list.argtypes = [vp, vp, vp, vp, i]
        L.orc_sphere_list.restype = i
        L.orc_sphere_walls.argtypes = [vp, vp]
        L.orc_sphere_counts.argtypes = [vp, vp]
        _bound.add(id(L))
    return L


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class OracleSphereWorld:
    """The oracle's spheres: the same surface as the CUDA library's SphereSimulation, plus the list's inspection.

    solve: 0 Jacobi, 1 Gauss-Seidel over the contact list run until done, 2 the same with `rounds` rounds a pass.
    grid: a SphereGrid, or None for every pair (Jacobi only).
    """

    def __init__(self, n, substeps, iterations, solve, grid, rounds=32, per_sphere=6, threads=False):
        if solve != 0 and grid is None:
            raise ValueError("Gauss-Seidel works over the grid's cells, and there is no grid")
        self.L = lib(threads)
        self.n = n
        self.capacity = n * per_sphere
        g = grid
        self.h = self.L.orc_sphere_create(n, substeps, iterations, solve, rounds, g.nx if g else 0, g.ny if g else 0,
                                          g.nz if g else 0, g.cell if g else 1.0, per_sphere)

    def close(self):
        if self.h:
            self.L.orc_sphere_destroy(self.h)
            self.h = None

    __del__ = close

    def set_field(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float32)
        assert a.shape == (self.n,)
        self.L.orc_sphere_set_field(self.h, FIELDS.index(name), _ptr(a))

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.n, np.float32)
        self.L.orc_sphere_get_field(self.h, FIELDS.index(name), _ptr(out))
        return out

    def set_params(self, bits, friction: bool) -> None:
        a = np.ascontiguousarray(bits, dtype=np.int32)
        self.L.orc_sphere_set_params(self.h, _ptr(a), int(bool(friction)))

    def set_shown(self, shown) -> None:
        a = np.ascontiguousarray(shown, dtype=np.float32)
        self.L.orc_sphere_set_shown(self.h, _ptr(a))

    def shown(self) -> np.ndarray:
        out = np.empty(self.n * SHOWN_STRIDE, np.float32)
        self.L.orc_sphere_shown(self.h, _ptr(out))
        return out

    def step(self, steps: int = 1):
        """Steps; returns the last step's (waits, rounds, most rounds, unlisted)."""
        report = np.zeros(4, np.int32)
        status = self.L.orc_sphere_step(self.h, steps, _ptr(report))
        if status != 0:
            raise RuntimeError("a pass is still open past its round limit")
        return tuple(int(v) for v in report)

    def contact_list(self):
        """The last substep's list in list order: pairs (k, 2), done marks (k,), impulses (k, 7)."""
        ab = np.zeros((self.capacity, 2), np.int32)
        done = np.zeros(self.capacity, np.int32)
        imp = np.zeros((self.capacity, IMPULSE_WORDS), np.float32)
        k = self.L.orc_sphere_list(self.h, _ptr(ab), _ptr(done), _ptr(imp), self.capacity)
        return ab[:k], done[:k], imp[:k]

    def walls(self) -> np.ndarray:
        out = np.empty(self.n * WALL_IMPULSE_WORDS, np.float32)
        self.L.orc_sphere_walls(self.h, _ptr(out))
        return out

    def counts(self) -> np.ndarray:
        out = np.zeros(3, np.int32)
        self.L.orc_sphere_counts(self.h, _ptr(out))
        return out
