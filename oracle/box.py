"""CPU ORACLE — test infrastructure only. ctypes binding of the C++ restatement in ``box_oracle.cpp``.

Used by tests/, ``__graft_entry__.smoke()`` (as the checker) and bench.py's CPU-baseline leg; never by the
product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

FIELDS = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw", "im", "hx", "hy", "hz", "shape"]
BUFFERS = {"pairs": (0, np.int32), "manifold": (1, np.float32), "impulses": (2, np.float32),
           "contacts": (3, np.int32), "lambda": (4, np.float32), "rub": (5, np.float32),
           "roll": (6, np.float32), "rounds": (7, np.int32)}

_libs: dict[bool, ctypes.CDLL] = {}


def build() -> None:
    """Compiles the oracle libraries with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(threads: bool = False) -> ctypes.CDLL:
    if threads not in _libs:
        name = "liborc_omp.so" if threads else "liborc.so"
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.orc_box_create.restype = vp
        L.orc_box_create.argtypes = [i, i, i, i, i, i, i, f, i]
        L.orc_box_destroy.argtypes = [vp]
        L.orc_box_set_reach.argtypes = [vp, i]
        L.orc_box_set_field.argtypes = [vp, i, vp]
        L.orc_box_get_field.argtypes = [vp, i, vp]
        L.orc_box_set_params.argtypes = [vp, vp]
        L.orc_box_set_shown.argtypes = [vp, vp]
        L.orc_box_get_shown.argtypes = [vp, vp]
        L.orc_box_step.argtypes = [vp, i, vp]
        L.orc_box_slots.argtypes = [vp]
        L.orc_box_slots.restype = i
        L.orc_box_buffer_words.argtypes = [vp, i]
        L.orc_box_buffer_words.restype = ctypes.c_long
        L.orc_box_buffer.argtypes = [vp, i]
        L.orc_box_buffer.restype = vp
        L.orc_collide.argtypes = [i, vp, vp, i, vp, vp]
        L.orc_threads.restype = i
        _libs[threads] = L
    return _libs[threads]


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class OracleBoxWorld:
    """The oracle's box/mixed world: the same start / step / state surface as the CUDA library's BoxSimulation."""

    def __init__(self, n, substeps, sweeps, symmetric, grid, threads=False, reach_cells=1):
        self.L = lib(threads)
        self.n = n
        g = grid
        self.h = self.L.orc_box_create(n, substeps, sweeps, int(bool(symmetric)), g.nx if g else 1,
                                       g.ny if g else 1, g.nz if g else 1, g.cell if g else 1.0,
                                       1 if g is not None else 0)
        self.L.orc_box_set_reach(self.h, int(reach_cells))

    def close(self):
        if self.h:
            self.L.orc_box_destroy(self.h)
            self.h = None

    __del__ = close

    def set_field(self, name, values):
        a = np.ascontiguousarray(values, dtype=np.float32)
        assert a.shape == (self.n,)
        self.L.orc_box_set_field(self.h, FIELDS.index(name), _ptr(a))

    def field(self, name) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float32)
        self.L.orc_box_get_field(self.h, FIELDS.index(name), _ptr(out))
        return out

    def set_params(self, bits):
        a = np.ascontiguousarray(bits, dtype=np.int32)
        assert a.shape == (18,)
        self.L.orc_box_set_params(self.h, _ptr(a))

    def set_shown(self, shown):
        a = np.ascontiguousarray(shown, dtype=np.float32)
        self.L.orc_box_set_shown(self.h, _ptr(a))

    def shown(self) -> np.ndarray:
        out = np.empty(20 * self.n, dtype=np.float32)
        self.L.orc_box_get_shown(self.h, _ptr(out))
        return out

    def step(self, steps=1) -> tuple:
        rep = np.zeros(5, dtype=np.int32)
        self.L.orc_box_step(self.h, steps, _ptr(rep))
        return tuple(int(v) for v in rep)

    @property
    def slots(self) -> int:
        return self.L.orc_box_slots(self.h)

    def buffer(self, name) -> np.ndarray:
        which, dt = BUFFERS[name]
        words = self.L.orc_box_buffer_words(self.h, which)
        if words == 0:
            return np.zeros(0, dtype=dt)
        addr = self.L.orc_box_buffer(self.h, which)
        return _array(addr, words, dt).copy()

    def touching_pairs(self):
        """The touching pairs of the last step, ascending: [(first, second, points)]."""
        c = self.buffer("contacts")
        slots = self.slots
        out = []
        for p in np.nonzero(c[:slots] >= 0)[0]:
            out.append((int(p // 32), int(c[p]), int(c[slots + p])))
        return out

    def touching_manifolds(self):
        """The manifolds (40 words each) of the last step's touching pairs, in ascending pair order."""
        c = self.buffer("contacts")
        m = self.buffer("manifold").reshape(-1, 40)
        return [m[p] for p in np.nonzero(c[:self.slots] >= 0)[0]]

    def touching_impulses(self):
        """The impulse records (28 words each) of the last step's touching pairs, in ascending pair order."""
        c = self.buffer("contacts")
        m = self.buffer("impulses").reshape(-1, 28)
        return [m[p] for p in np.nonzero(c[:self.slots] >= 0)[0]]

    def candidate_pairs(self):
        """The broad phase's candidate pairs of the last step, ascending: an (m, 2) int array."""
        pairs = self.buffer("pairs").reshape(-1, 2)
        keep = pairs[:, 1] >= 0
        return pairs[keep]


def _array(addr, words, dt):
    ctype = ctypes.c_int32 if dt == np.int32 else ctypes.c_float
    return np.ctypeslib.as_array((ctype * words).from_address(addr))


def collide(fields18: list, param_bits, pairs, threads=False) -> np.ndarray:
    """The collide pass alone over ``pairs`` (flat first, second, ...): manifolds, 40 words each."""
    L = lib(threads)
    arrs = [np.ascontiguousarray(f, dtype=np.float32) for f in fields18]
    ptrs = (ctypes.c_void_p * 18)(*[a.ctypes.data for a in arrs])
    pb = np.ascontiguousarray(param_bits, dtype=np.int32)
    pr = np.ascontiguousarray(pairs, dtype=np.int32)
    npairs = len(pr) // 2
    out = np.zeros(40 * npairs, dtype=np.float32)
    L.orc_collide(len(arrs[0]), ctypes.cast(ptrs, ctypes.c_void_p), _ptr(pb), npairs, _ptr(pr), _ptr(out))
    return out
