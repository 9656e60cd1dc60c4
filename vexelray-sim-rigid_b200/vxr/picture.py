"""The picture of a step: the reference's fragment shaders (gui/SphereShader.java, gui/BoxShader.java over
gui/Picture.java) as CUDA kernels (include/vxr.h, vxr_picture), one thread a pixel, written into a headless RGB
buffer; and the camera RigidView.show (gui/RigidView.java:63-74) puts in the push constants."""
from __future__ import annotations

import ctypes
import math

import numpy as np

from ._lib import Camera, VxrError, lib, ptr

SPHERES, BOXES = 0, 1


def _normalise(x, y, z):
    length = math.sqrt(x * x + y * y + z * z)
    return (x / length, y / length, z / length)


def orbit_camera(extent, pose, alpha=1.0, squash=0.0, aspect=1.0) -> Camera:
    """RigidView.show's camera: an orbit pose (x, y, z) about a box scaled so its longest side is two units across,
    centred on the origin, turned into the simulation's metres; right is (f.z, 0, -f.x) normalised, up is f x r."""
    longest = max(extent)
    scale = longest / 2
    eye = [extent[a] / 2 + pose[a] * scale for a in range(3)]
    forward = _normalise(-pose[0], -pose[1], -pose[2])
    right = _normalise(forward[2], 0.0, -forward[0])
    up = (forward[1] * right[2] - forward[2] * right[1], forward[2] * right[0] - forward[0] * right[2],
          forward[0] * right[1] - forward[1] * right[0])
    return camera(eye, right, up, forward, aspect, alpha, extent, squash)


def camera(eye, right, up, forward, aspect, alpha, extent, squash) -> Camera:
    c = Camera()
    for a in range(3):
        c.eye[a], c.right[a], c.up[a], c.forward[a], c.extent[a] = eye[a], right[a], up[a], forward[a], extent[a]
    c.aspect, c.alpha, c.squash = aspect, alpha, squash
    return c


def push_words(c: Camera, count: int) -> np.ndarray:
    """The 19 push-constant floats of Picture.push for this camera and `count` bodies."""
    return np.array(list(c.eye) + list(c.right) + list(c.up) + list(c.forward) + [c.aspect, c.alpha, float(count)]
                    + list(c.extent) + [c.squash], dtype=np.float32)


def draw(shape: int, shown, count: int, cam: Camera, width: int, height: int, rgb, stream=None) -> None:
    """`count` bodies from `shown` (a device pointer or a CUDA tensor) drawn into `rgb` (a device pointer or a CUDA
    float32 tensor of height x width x 3) on `stream` (a CUDA stream handle; None for the default stream)."""
    src = shown.data_ptr() if hasattr(shown, "data_ptr") else shown
    dst = rgb.data_ptr() if hasattr(rgb, "data_ptr") else rgb
    if hasattr(rgb, "numel") and rgb.numel() < width * height * 3:
        raise ValueError("rgb holds fewer than width * height * 3 floats")
    rc = lib().vxr_picture(shape, src, count, ctypes.byref(cam), width, height, dst, stream)
    if rc:
        raise VxrError(rc, "picture")


def draw_frame(frame, cam: Camera, width: int, height: int, rgb, stream=None) -> None:
    """A ring frame (vxr.shown_ring) drawn once its slot is complete: the stream waits on the slot's event first."""
    rc = lib().vxr_ring_wait(ctypes.byref(frame), stream)
    if rc:
        raise VxrError(rc, "wait")
    draw(frame.shape, frame.data, frame.bodies, cam, width, height, rgb, stream)


def draw_host(shape: int, shown: np.ndarray, count: int, cam: Camera, width: int, height: int) -> np.ndarray:
    """The same from and into host memory: the picture as (height, width, 3) float32, row 0 the top."""
    s = np.ascontiguousarray(shown, np.float32)
    if s.size == 0:
        s = np.zeros(1, np.float32)
    out = np.empty((height, width, 3), np.float32)
    rc = lib().vxr_picture_host(shape, ptr(s), count, ctypes.byref(cam), width, height, ptr(out))
    if rc:
        raise VxrError(rc, "picture")
    return out


def write_ppm(path: str, rgb: np.ndarray) -> None:
    """A picture written as a binary PPM, each channel clamped to [0, 1] and scaled to 0-255."""
    h, w, _ = rgb.shape
    b = (np.clip(rgb, 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(f"P6\n{w} {h}\n255\n".encode())
        f.write(b.tobytes())
