"""The picture's hand-off: the reference's ShownRing (gui/ShownRing.java:37-177) over the library's native ring
(include/vxr.h, vxr_ring_*), its slots in device memory, a CUDA event for each slot's timeline value."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import Frame, VxrError, lib, ptr

SPHERES, BOXES = 0, 1
SLOTS = 3


class ShownRing:
    def __init__(self, device: int = 0):
        self.h = lib().vxr_ring_create(device)

    def install(self, shape: int, bodies: int, extent=(1.0, 1.0, 1.0)) -> int:
        e = np.ascontiguousarray(extent, np.float64)
        gid = lib().vxr_ring_install(self.h, shape, bodies, ptr(e))
        if gid < 0:
            raise VxrError(-gid, "install")
        return gid

    def back(self) -> int:
        return lib().vxr_ring_back(self.h)

    def publish(self, step: int, finished_ns: int) -> None:
        rc = lib().vxr_ring_publish(self.h, step, finished_ns)
        if rc:
            raise VxrError(rc, "publish: no generation installed")

    def keep(self, world, step: int) -> None:
        """Keeps a box or sphere world's `shown` as step `step` (on the world's stream) and publishes it."""
        words = ctypes.c_int64(0)
        if hasattr(world, "_h"):  # a SphereSimulation
            src = lib().vxr_sphere_shown_device(world._h, ctypes.byref(words))
            stream = world.stream()
        else:
            src = lib().vxr_box_shown_device(world.h, ctypes.byref(words))
            stream = world.stream
        rc = lib().vxr_ring_keep(self.h, src, words.value, stream, step)
        if rc:
            raise VxrError(rc, lib().vxr_ring_error(self.h).decode())

    def take(self):
        """The newest finished step as the front (a Frame), or None before any step has been published."""
        f = Frame()
        rc = lib().vxr_ring_take(self.h, ctypes.byref(f))
        if rc == 1:
            return None
        if rc:
            raise VxrError(rc, "take")
        return f

    @staticmethod
    def read(frame) -> np.ndarray:
        out = np.empty(frame.words, np.float32)
        rc = lib().vxr_ring_read(ctypes.byref(frame), ptr(out))
        if rc:
            raise VxrError(rc, "read")
        return out

    def retired(self) -> list:
        ids = np.zeros(64, np.int64)
        n = lib().vxr_ring_retired(self.h, ptr(ids), len(ids))
        return [int(i) for i in ids[:n]]

    def live(self) -> list:
        ids = np.zeros(64, np.int64)
        n = lib().vxr_ring_live(self.h, ptr(ids), len(ids))
        return [int(i) for i in ids[:n]]

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().vxr_ring_destroy(self.h)
            self.h = None

    __del__ = close
