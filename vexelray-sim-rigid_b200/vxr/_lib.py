"""ctypes binding of libvxr.so, the C-ABI declared in include/vxr.h.

The library is built in-tree (vexelray-sim-rigid_b200/csrc/Makefile). Loading it needs no GPU; stepping a world
does, and fails loudly (an exception carrying the library's status and message) when there is none: there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvxr.so")

VXR_OK, VXR_EINVAL, VXR_ECAPACITY, VXR_EROUNDS, VXR_ENONFINITE, VXR_ETIMEOUT, VXR_ECUDA = range(7)
STATUS_NAMES = {0: "VXR_OK", 1: "VXR_EINVAL", 2: "VXR_ECAPACITY", 3: "VXR_EROUNDS", 4: "VXR_ENONFINITE",
                5: "VXR_ETIMEOUT", 6: "VXR_ECUDA"}

#: Every symbol include/vxr.h declares (checked by the CPU test suite).
SYMBOLS = ["vxr_version", "vxr_box_make_params", "vxr_box_make_grid", "vxr_box_create", "vxr_box_destroy",
           "vxr_box_error", "vxr_box_start", "vxr_box_load_state", "vxr_box_params", "vxr_box_step",
           "vxr_box_step_async", "vxr_box_sync", "vxr_box_stream", "vxr_box_state", "vxr_box_state_async", "vxr_box_state_wait", "vxr_box_read_shown",
           "vxr_box_touching", "vxr_box_candidates", "vxr_box_walls", "vxr_box_colour_waves", "vxr_collide",
           "vxr_box_launches", "vxr_box_profile", "vxr_box_activity", "vxr_box_trace", "vxr_box_broadphase_static",
           "vxr_box_measure", "vxr_box_list_kernel", "vxr_box_wait_limit", "vxr_box_islands", "vxr_box_paths", "vxr_box_residuals", "vxr_box_residual_parts", "vxr_box_create_batch", "vxr_box_scene_params",
           "vxr_box_scenes", "vxr_box_step_graph", "vxr_mlp_create", "vxr_mlp_destroy", "vxr_mlp_error",
           "vxr_mlp_set", "vxr_mlp_get", "vxr_mlp_forward", "vxr_mlp_gradients", "vxr_mlp_train", "vxr_box_learned", "vxr_box_learned_given", "vxr_box_first_substeps",
           "vxr_box_features", "vxr_box_diagnostics", "vxr_box_contact_errors", "vxr_sphere_diagnostics", "vxr_ring_create", "vxr_ring_destroy",
           "vxr_ring_error", "vxr_ring_install", "vxr_ring_back", "vxr_ring_publish", "vxr_ring_keep", "vxr_ring_take",
           "vxr_ring_wait", "vxr_ring_read", "vxr_ring_retired", "vxr_ring_live", "vxr_box_shown_device",
           "vxr_sphere_shown_device", "vxr_picture", "vxr_picture_host",
           "vxr_sphere_make_params", "vxr_sphere_make_grid", "vxr_sphere_create", "vxr_sphere_destroy",
           "vxr_sphere_error", "vxr_sphere_start", "vxr_sphere_load_state", "vxr_sphere_params", "vxr_sphere_friction",
           "vxr_sphere_round_limit",
           "vxr_sphere_step", "vxr_sphere_step_async", "vxr_sphere_sync", "vxr_sphere_stream", "vxr_sphere_state",
           "vxr_sphere_field", "vxr_sphere_read_shown", "vxr_sphere_contacts", "vxr_sphere_walls",
           "vxr_sphere_counts", "vxr_sphere_blocks", "vxr_sphere_launches"]


class VxrError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("cell", ctypes.c_float)]


class BoxConfig(ctypes.Structure):
    _fields_ = [("bodies", ctypes.c_int32), ("substeps", ctypes.c_int32), ("sweeps", ctypes.c_int32),
                ("symmetric", ctypes.c_int32), ("grid", Grid), ("reach_cells", ctypes.c_int32),
                ("max_pairs", ctypes.c_int32), ("device", ctypes.c_int32), ("schedule", ctypes.c_int32),
                ("solve_blocks_per_sm", ctypes.c_int32)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("scenes", ctypes.c_int32), ("bodies", ctypes.c_void_p), ("grids", ctypes.c_void_p),
                ("substeps", ctypes.c_int32), ("sweeps", ctypes.c_int32), ("symmetric", ctypes.c_int32),
                ("max_pairs", ctypes.c_int32), ("device", ctypes.c_int32), ("schedule", ctypes.c_int32),
                ("solve_blocks_per_sm", ctypes.c_int32)]


class BoxReport(ctypes.Structure):
    _fields_ = [("touching", ctypes.c_int32), ("points", ctypes.c_int32), ("rounds", ctypes.c_int32),
                ("unplaced", ctypes.c_int32), ("unlisted", ctypes.c_int32), ("most_rounds", ctypes.c_int32),
                ("unplaced_total", ctypes.c_int64), ("unlisted_total", ctypes.c_int64), ("status", ctypes.c_int32),
                ("steps", ctypes.c_int32)]


class Diag(ctypes.Structure):
    """vxr_box_diag and vxr_sphere_diag: the same layout (the overlap words are named for the box's)."""
    _fields_ = [("kinetic", ctypes.c_double), ("rotational", ctypes.c_double), ("potential", ctypes.c_double),
                ("momentum", ctypes.c_double * 3), ("angular", ctypes.c_double * 3),
                ("max_penetration", ctypes.c_double), ("max_wall", ctypes.c_double), ("max_speed", ctypes.c_double),
                ("broken", ctypes.c_int32), ("pad", ctypes.c_int32)]


class Frame(ctypes.Structure):
    _fields_ = [("generation", ctypes.c_int64), ("step", ctypes.c_int64), ("finished_ns", ctypes.c_int64),
                ("words", ctypes.c_int64), ("slot", ctypes.c_int32), ("shape", ctypes.c_int32),
                ("bodies", ctypes.c_int32), ("pad", ctypes.c_int32), ("extent", ctypes.c_double * 3),
                ("data", ctypes.c_void_p), ("event", ctypes.c_void_p)]


class Camera(ctypes.Structure):
    """vxr_camera: Picture.push's words (gui/Picture.java:202-216) as a struct."""
    _fields_ = [("eye", ctypes.c_float * 3), ("right", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("forward", ctypes.c_float * 3), ("aspect", ctypes.c_float), ("alpha", ctypes.c_float),
                ("extent", ctypes.c_float * 3), ("squash", ctypes.c_float)]


class SphereConfig(ctypes.Structure):
    _fields_ = [("spheres", ctypes.c_int32), ("substeps", ctypes.c_int32), ("iterations", ctypes.c_int32),
                ("solve", ctypes.c_int32), ("rounds", ctypes.c_int32), ("contacts_per_sphere", ctypes.c_int32),
                ("grid", Grid), ("device", ctypes.c_int32), ("blocks", ctypes.c_int32), ("cluster", ctypes.c_int32)]


class SphereReport(ctypes.Structure):
    _fields_ = [("waits", ctypes.c_int32), ("rounds", ctypes.c_int32), ("most_rounds", ctypes.c_int32),
                ("unlisted", ctypes.c_int32), ("waits_total", ctypes.c_int64), ("rounds_total", ctypes.c_int64),
                ("most_rounds_total", ctypes.c_int32), ("status", ctypes.c_int32),
                ("unlisted_total", ctypes.c_int64), ("listed", ctypes.c_int32), ("pad", ctypes.c_int32)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built: run `make -C vexelray-sim-rigid_b200/csrc` "
                          "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, f64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_float
        L.vxr_version.restype = ctypes.c_char_p
        L.vxr_box_make_params.argtypes = [f64] * 11 + [vp]
        L.vxr_box_make_params.restype = i32
        L.vxr_box_make_grid.argtypes = [f64] * 5 + [ctypes.POINTER(Grid)]
        L.vxr_box_make_grid.restype = i32
        L.vxr_box_create.argtypes = [ctypes.POINTER(BoxConfig), ctypes.POINTER(i32)]
        L.vxr_box_create.restype = vp
        L.vxr_box_destroy.argtypes = [vp]
        L.vxr_box_error.argtypes = [vp]
        L.vxr_box_error.restype = ctypes.c_char_p
        L.vxr_box_start.argtypes = [vp] + [vp] * 11 + [vp]
        L.vxr_box_start.restype = i32
        L.vxr_box_load_state.argtypes = [vp, vp, vp]
        L.vxr_box_load_state.restype = i32
        L.vxr_box_params.argtypes = [vp, vp]
        L.vxr_box_params.restype = i32
        L.vxr_box_step.argtypes = [vp, i32, ctypes.POINTER(BoxReport)]
        L.vxr_box_step.restype = i32
        L.vxr_box_step_async.argtypes = [vp, i32]
        L.vxr_box_step_async.restype = i32
        L.vxr_box_sync.argtypes = [vp, ctypes.POINTER(BoxReport)]
        L.vxr_box_sync.restype = i32
        L.vxr_box_stream.argtypes = [vp]
        L.vxr_box_stream.restype = vp
        L.vxr_box_state.argtypes = [vp, vp]
        L.vxr_box_state.restype = i32
        L.vxr_box_state_async.argtypes = [vp, vp, i32]
        L.vxr_box_state_async.restype = i32
        L.vxr_box_state_wait.argtypes = [vp, i32]
        L.vxr_box_state_wait.restype = i32
        L.vxr_box_read_shown.argtypes = [vp, vp]
        L.vxr_box_read_shown.restype = i32
        L.vxr_box_touching.argtypes = [vp, vp, vp, vp, vp, vp, i32]
        L.vxr_box_touching.restype = i32
        L.vxr_box_candidates.argtypes = [vp, vp, i32]
        L.vxr_box_candidates.restype = i32
        L.vxr_box_walls.argtypes = [vp, vp, vp, vp]
        L.vxr_box_walls.restype = i32
        L.vxr_box_colour_waves.argtypes = [vp]
        L.vxr_box_colour_waves.restype = i32
        L.vxr_box_launches.argtypes = [vp]
        L.vxr_box_launches.restype = ctypes.c_longlong
        L.vxr_box_profile.argtypes = [vp, i32, vp]
        L.vxr_box_profile.restype = i32
        L.vxr_box_activity.argtypes = [vp, vp]
        L.vxr_box_activity.restype = i32
        L.vxr_box_trace.argtypes = [vp, i32, vp, i32]
        L.vxr_box_trace.restype = i32
        L.vxr_box_measure.argtypes = [vp, i32, i32, i32, ctypes.c_float]
        L.vxr_box_measure.restype = i32
        L.vxr_box_list_kernel.argtypes = [vp, i32]
        L.vxr_box_list_kernel.restype = i32
        L.vxr_box_wait_limit.argtypes = [vp, ctypes.c_int64]
        L.vxr_box_wait_limit.restype = i32
        L.vxr_box_islands.argtypes = [vp, i32]
        L.vxr_box_islands.restype = i32
        L.vxr_box_paths.argtypes = [vp, vp]
        L.vxr_box_paths.restype = i32
        L.vxr_box_residuals.argtypes = [vp, vp, i32, vp]
        L.vxr_box_residuals.restype = i32
        L.vxr_box_residual_parts.argtypes = [vp, vp, vp, i32]
        L.vxr_box_residual_parts.restype = i32
        L.vxr_box_broadphase_static.argtypes = [i32, vp, Grid, i32, f32, vp, vp, i32, vp, vp]
        L.vxr_box_broadphase_static.restype = i32
        L.vxr_collide.argtypes = [i32, vp, vp, i32, vp, vp]
        L.vxr_collide.restype = i32
        L.vxr_box_create_batch.argtypes = [ctypes.POINTER(BatchConfig), ctypes.POINTER(i32)]
        L.vxr_box_create_batch.restype = vp
        L.vxr_box_scene_params.argtypes = [vp, vp]
        L.vxr_box_scene_params.restype = i32
        L.vxr_box_scenes.argtypes = [vp, vp]
        L.vxr_box_scenes.restype = i32
        L.vxr_box_step_graph.argtypes = [vp, i32]
        L.vxr_box_step_graph.restype = i32
        L.vxr_mlp_create.argtypes = [i32, ctypes.c_uint64, ctypes.POINTER(i32)]
        L.vxr_mlp_create.restype = vp
        L.vxr_mlp_destroy.argtypes = [vp]
        L.vxr_mlp_error.argtypes = [vp]
        L.vxr_mlp_error.restype = ctypes.c_char_p
        L.vxr_mlp_set.argtypes = [vp, vp, vp, vp]
        L.vxr_mlp_set.restype = i32
        L.vxr_mlp_get.argtypes = [vp, vp, vp, vp]
        L.vxr_mlp_get.restype = i32
        L.vxr_mlp_forward.argtypes = [vp, vp, i32, vp]
        L.vxr_mlp_forward.restype = i32
        L.vxr_mlp_gradients.argtypes = [vp, vp, vp, i32, vp, vp]
        L.vxr_mlp_gradients.restype = i32
        L.vxr_mlp_train.argtypes = [vp, vp, vp, i32, i32, i32, ctypes.c_float, ctypes.c_uint64, vp]
        L.vxr_mlp_train.restype = i32
        L.vxr_box_learned.argtypes = [vp, vp, i32]
        L.vxr_box_learned.restype = i32
        L.vxr_box_first_substeps.argtypes = [vp, i32, i32]
        L.vxr_box_first_substeps.restype = i32
        L.vxr_box_learned_given.argtypes = [vp, vp, i32, i32]
        L.vxr_box_learned_given.restype = i32
        L.vxr_box_features.argtypes = [vp, vp, vp, i32, ctypes.POINTER(i32)]
        L.vxr_box_features.restype = i32
        L.vxr_box_diagnostics.argtypes = [vp, ctypes.POINTER(Diag)]
        L.vxr_box_diagnostics.restype = i32
        L.vxr_box_contact_errors.argtypes = [vp, vp, i32]
        L.vxr_box_contact_errors.restype = i32
        L.vxr_sphere_diagnostics.argtypes = [vp, ctypes.POINTER(Diag)]
        L.vxr_sphere_diagnostics.restype = i32
        L.vxr_ring_create.argtypes = [i32]
        L.vxr_ring_create.restype = vp
        L.vxr_ring_destroy.argtypes = [vp]
        L.vxr_ring_error.argtypes = [vp]
        L.vxr_ring_error.restype = ctypes.c_char_p
        L.vxr_ring_install.argtypes = [vp, i32, i32, vp]
        L.vxr_ring_install.restype = ctypes.c_int64
        L.vxr_ring_back.argtypes = [vp]
        L.vxr_ring_back.restype = i32
        L.vxr_ring_publish.argtypes = [vp, ctypes.c_int64, ctypes.c_int64]
        L.vxr_ring_publish.restype = i32
        L.vxr_ring_keep.argtypes = [vp, vp, ctypes.c_int64, vp, ctypes.c_int64]
        L.vxr_ring_keep.restype = i32
        L.vxr_ring_take.argtypes = [vp, ctypes.POINTER(Frame)]
        L.vxr_ring_take.restype = i32
        L.vxr_ring_wait.argtypes = [ctypes.POINTER(Frame), vp]
        L.vxr_ring_wait.restype = i32
        L.vxr_ring_read.argtypes = [ctypes.POINTER(Frame), vp]
        L.vxr_ring_read.restype = i32
        L.vxr_ring_retired.argtypes = [vp, vp, i32]
        L.vxr_ring_retired.restype = i32
        L.vxr_ring_live.argtypes = [vp, vp, i32]
        L.vxr_ring_live.restype = i32
        L.vxr_box_shown_device.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.vxr_box_shown_device.restype = vp
        L.vxr_sphere_shown_device.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.vxr_sphere_shown_device.restype = vp
        L.vxr_picture.argtypes = [i32, vp, i32, ctypes.POINTER(Camera), i32, i32, vp, vp]
        L.vxr_picture.restype = i32
        L.vxr_picture_host.argtypes = [i32, vp, i32, ctypes.POINTER(Camera), i32, i32, vp]
        L.vxr_picture_host.restype = i32
        L.vxr_sphere_make_params.argtypes = [f64] * 8 + [i32] + [f64] * 4 + [vp]
        L.vxr_sphere_make_params.restype = i32
        L.vxr_sphere_make_grid.argtypes = [f64] * 4 + [ctypes.POINTER(Grid)]
        L.vxr_sphere_make_grid.restype = i32
        L.vxr_sphere_create.argtypes = [ctypes.POINTER(SphereConfig), ctypes.POINTER(i32)]
        L.vxr_sphere_create.restype = vp
        L.vxr_sphere_destroy.argtypes = [vp]
        L.vxr_sphere_error.argtypes = [vp]
        L.vxr_sphere_error.restype = ctypes.c_char_p
        L.vxr_sphere_start.argtypes = [vp] + [vp] * 8 + [vp]
        L.vxr_sphere_start.restype = i32
        L.vxr_sphere_load_state.argtypes = [vp, vp, vp]
        L.vxr_sphere_load_state.restype = i32
        L.vxr_sphere_params.argtypes = [vp, vp]
        L.vxr_sphere_params.restype = i32
        L.vxr_sphere_friction.argtypes = [vp, i32]
        L.vxr_sphere_friction.restype = i32
        L.vxr_sphere_round_limit.argtypes = [vp, i32]
        L.vxr_sphere_round_limit.restype = i32
        L.vxr_sphere_step.argtypes = [vp, i32, ctypes.POINTER(SphereReport)]
        L.vxr_sphere_step.restype = i32
        L.vxr_sphere_step_async.argtypes = [vp, i32]
        L.vxr_sphere_step_async.restype = i32
        L.vxr_sphere_sync.argtypes = [vp, ctypes.POINTER(SphereReport)]
        L.vxr_sphere_sync.restype = i32
        L.vxr_sphere_stream.argtypes = [vp]
        L.vxr_sphere_stream.restype = vp
        L.vxr_sphere_state.argtypes = [vp, vp]
        L.vxr_sphere_state.restype = i32
        L.vxr_sphere_field.argtypes = [vp, i32, vp]
        L.vxr_sphere_field.restype = i32
        L.vxr_sphere_read_shown.argtypes = [vp, vp]
        L.vxr_sphere_read_shown.restype = i32
        L.vxr_sphere_contacts.argtypes = [vp, vp, vp, vp, i32, ctypes.POINTER(i32)]
        L.vxr_sphere_contacts.restype = i32
        L.vxr_sphere_walls.argtypes = [vp, vp]
        L.vxr_sphere_walls.restype = i32
        L.vxr_sphere_counts.argtypes = [vp, vp]
        L.vxr_sphere_counts.restype = i32
        L.vxr_sphere_blocks.argtypes = [vp]
        L.vxr_sphere_blocks.restype = i32
        L.vxr_sphere_launches.argtypes = [vp]
        L.vxr_sphere_launches.restype = ctypes.c_longlong
        _lib = L
    return _lib


def ptr(a) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def ptr_array(arrays) -> ctypes.Array:
    return (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
