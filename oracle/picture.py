"""CPU ORACLE — test infrastructure only. ctypes binding of the C++ restatement in ``picture_oracle.cpp``: the
reference's sphere and box fragment shaders (gui/SphereShader.java, gui/BoxShader.java over gui/Picture.java), one
pixel at a time.

Used by tests/ and ``__graft_entry__.smoke()`` as the checker; never by the product path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import box

SPHERES, BOXES = 0, 1
_bound: set = set()


def lib() -> ctypes.CDLL:
    L = box.lib(False)
    if id(L) not in _bound:
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.orc_picture.argtypes = [i, vp, vp, i, i, i, i, vp]
        _bound.add(id(L))
    return L


def push(eye, right, up, forward, aspect, alpha, count, extent, squash) -> np.ndarray:
    """Picture.push (gui/Picture.java:202-216): the 19 push-constant floats of one frame."""
    words = list(eye) + list(right) + list(up) + list(forward) + [aspect, alpha, count] + list(extent) + [squash]
    return np.array(words, dtype=np.float32)


def picture(shape: int, shown: np.ndarray, push_words: np.ndarray, width: int, height: int, rows=None) -> np.ndarray:
    """The picture, (height, width, 3) float32, row 0 the top; or only `rows` (a range) of it."""
    rows = range(height) if rows is None else rows
    shown = np.ascontiguousarray(shown, dtype=np.float32)
    if shown.size == 0:
        shown = np.zeros(1, np.float32)
    p = np.ascontiguousarray(push_words, dtype=np.float32)
    out = np.zeros((len(rows), width, 3), np.float32)
    lib().orc_picture(shape, shown.ctypes.data, p.ctypes.data, width, height, rows.start, len(rows), out.ctypes.data)
    return out
