"""Spheres in a box on the B200: the reference's SphereSimulation (gui/SphereSimulation.java:33-295) over the C-ABI
(include/vxr.h, libvxr.so).

    sim = SphereSimulation(n, substeps, iterations, spheres.covering(sx, sy, sz, widest), GAUSS_SEIDEL_BY_CONTACT)
    sim.start(x, y, z, u, v, w, r, im, spheres.params(h, 0, -9.81, 0, sx, sy, sz, 1, True, 0.2, 0.5, 0.5))
    report = sim.step_and_wait()          # SphereStepper.Report: waits, rounds, most rounds, unlisted
    x, y, z, u, v, w, ax, ay, az = sim.state()

Every call goes to the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from collections import namedtuple

import numpy as np

from . import spheres as S
from ._lib import Diag, Grid, SphereConfig, SphereReport, VxrError, lib, ptr, ptr_array

Report = namedtuple("Report", "waits rounds most_rounds unlisted")


class SphereSimulation:
    """One world of spheres on one GPU. Not thread-safe: one world, one thread, as the reference's stepper."""

    def __init__(self, spheres: int, substeps: int, iterations: int, grid: S.SphereGrid | None,
                 solve: int = S.JACOBI, rounds: int = S.ROUNDS, contacts_per_sphere: int = S.CONTACTS_PER_SPHERE,
                 device: int = 0, blocks: int = 0, cluster: int = 0):
        L = lib()
        cfg = SphereConfig()
        cfg.spheres, cfg.substeps, cfg.iterations, cfg.solve = spheres, substeps, iterations, solve
        cfg.rounds, cfg.contacts_per_sphere, cfg.device, cfg.blocks = rounds, contacts_per_sphere, device, blocks
        cfg.cluster = cluster
        if grid is not None:
            cfg.grid = Grid(grid.nx, grid.ny, grid.nz, grid.cell)
        status = ctypes.c_int32(0)
        self._h = L.vxr_sphere_create(ctypes.byref(cfg), ctypes.byref(status))
        if not self._h:
            raise VxrError(status.value, "vxr_sphere_create")
        self.n = spheres
        self.capacity = spheres * contacts_per_sphere
        self.solve = solve
        self.last_report = None
        self.totals = None

    # -- the reference's calls ----------------------------------------------------------------------------------
    def _check(self, status: int) -> None:
        if status != 0:
            raise VxrError(status, lib().vxr_sphere_error(self._h).decode())

    def start(self, x, y, z, u, v, w, r, im, params) -> None:
        arrays = [np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z, u, v, w, r, im)]
        for a in arrays:
            if a.shape != (self.n,):
                raise ValueError("every array is as long as the sphere count")
        p = np.ascontiguousarray(params, dtype=np.int32)
        self._check(lib().vxr_sphere_start(self._h, *[ptr(a) for a in arrays], ptr(p)))

    def load_state(self, fields: dict, params) -> None:
        """The test fixture's start: any of the 24 fields by name, the rest zero (qw one)."""
        keep = [np.ascontiguousarray(fields[name], dtype=np.float32) if name in fields else None
                for name in S.FIELDS]
        table = (ctypes.c_void_p * 24)(*[a.ctypes.data if a is not None else None for a in keep])
        p = np.ascontiguousarray(params, dtype=np.int32)
        self._check(lib().vxr_sphere_load_state(self._h, table, ptr(p)))

    def params(self, params) -> None:
        p = np.ascontiguousarray(params, dtype=np.int32)
        self._check(lib().vxr_sphere_params(self._h, ptr(p)))

    def friction(self, on: bool) -> None:
        self._check(lib().vxr_sphere_friction(self._h, int(bool(on))))

    def round_limit(self, rounds: int = 0) -> None:
        """The rounds a pass run until done may take before the step is an error (VXR_EROUNDS); 0: the
        reference's limit, the list's capacity plus two cycles."""
        self._check(lib().vxr_sphere_round_limit(self._h, int(rounds)))

    def step_and_wait(self, steps: int = 1) -> Report:
        r = SphereReport()
        self._check(lib().vxr_sphere_step(self._h, steps, ctypes.byref(r)))
        self.last_report = Report(r.waits, r.rounds, r.most_rounds, r.unlisted)
        self.totals = Report(r.waits_total, r.rounds_total, r.most_rounds_total, r.unlisted_total)
        return self.last_report

    step = step_and_wait

    def step_async(self, steps: int = 1) -> None:
        self._check(lib().vxr_sphere_step_async(self._h, steps))

    def sync(self) -> Report:
        r = SphereReport()
        self._check(lib().vxr_sphere_sync(self._h, ctypes.byref(r)))
        self.last_report = Report(r.waits, r.rounds, r.most_rounds, r.unlisted)
        self.totals = Report(r.waits_total, r.rounds_total, r.most_rounds_total, r.unlisted_total)
        return self.last_report

    def state(self, out=None):
        """x y z u v w ax ay az; into `out` (9 float32 arrays of n, e.g. in pinned memory) when given."""
        if out is None:
            out = [np.empty(self.n, np.float32) for _ in range(9)]
        elif len(out) != 9 or any(a.dtype != np.float32 or a.shape != (self.n,) or not a.flags.c_contiguous
                                  for a in out):
            raise ValueError(f"out holds 9 contiguous float32 arrays of {self.n}")
        self._check(lib().vxr_sphere_state(self._h, ptr_array(out)))
        return out

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.n, np.float32)
        self._check(lib().vxr_sphere_field(self._h, S.FIELD[name], ptr(out)))
        return out

    def read_shown(self) -> np.ndarray:
        out = np.empty(self.n * S.SHOWN_STRIDE, np.float32)
        self._check(lib().vxr_sphere_read_shown(self._h, ptr(out)))
        return out

    shown = read_shown

    def stream(self) -> int:
        return lib().vxr_sphere_stream(self._h)

    def gpu_diagnostics(self) -> S.Diagnostics:
        """SphereDiagnostics computed on the GPU (vxr_sphere_diagnostics)."""
        d = Diag()
        self._check(lib().vxr_sphere_diagnostics(self._h, ctypes.byref(d)))
        return S.Diagnostics(d.max_penetration, d.max_wall, d.kinetic, d.rotational, d.potential, tuple(d.momentum),
                             tuple(d.angular), d.max_speed, bool(d.broken))

    def blocks(self) -> int:
        return lib().vxr_sphere_blocks(self._h)

    def launches(self) -> int:
        return lib().vxr_sphere_launches(self._h)

    # -- inspection -----------------------------------------------------------------------------------------------
    def contact_list(self):
        """The last substep's list in list order: pairs (k, 2), done marks (k,), impulses (k, 7)."""
        ab = np.zeros((self.capacity, 2), np.int32)
        done = np.zeros(self.capacity, np.int32)
        imp = np.zeros((self.capacity, S.IMPULSE_WORDS), np.float32)
        k = ctypes.c_int32(0)
        self._check(lib().vxr_sphere_contacts(self._h, ptr(ab), ptr(done), ptr(imp), self.capacity,
                                              ctypes.byref(k)))
        m = min(k.value, self.capacity)
        return ab[:m], done[:m], imp[:m]

    def walls(self) -> np.ndarray:
        out = np.empty(self.n * S.WALL_IMPULSE_WORDS, np.float32)
        self._check(lib().vxr_sphere_walls(self._h, ptr(out)))
        return out

    def counts(self) -> np.ndarray:
        out = np.zeros(3, np.int32)
        self._check(lib().vxr_sphere_counts(self._h, ptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().vxr_sphere_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def make_params(h, gx, gy, gz, sx, sy, sz, omega, averaged, restitution=0.0, mu_static=0.0, mu_kinetic=0.0,
                mu_rolling=0.0) -> np.ndarray:
    """Spheres.params through the C-ABI (the library's own validation)."""
    out = np.zeros(S.PARAM_COUNT, np.int32)
    status = lib().vxr_sphere_make_params(h, gx, gy, gz, sx, sy, sz, omega, int(bool(averaged)), restitution,
                                          mu_static, mu_kinetic, mu_rolling, ptr(out))
    if status != 0:
        raise VxrError(status, "bad sphere parameters")
    return out
