"""BoxSimulation: the reference's box/mixed simulation API, on the B200 through the C-ABI.

Mirrors gui/BoxSimulation.java (vexelray-sim-rigid-gui/src/main/java/dev/vexelray/sim/rigid/gui/BoxSimulation.java):
``start`` :77-108, ``params`` :111-113, ``step_and_wait`` :115-142, ``last`` :145-147, ``state`` :153-160,
``read_shown`` :163-165, ``close`` :183-188; and the step shape of core/box/BoxStep.java:81-162. Every call goes
through libvxr.so; nothing here computes the step.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import boxes as B
from ._lib import BatchConfig, BoxConfig, BoxReport, Diag, Grid, VxrError, lib, ptr, ptr_array

STATE_FIELDS = ["x", "y", "z", "u", "v", "w", "lx", "ly", "lz", "qx", "qy", "qz", "qw"]
ALL_FIELDS = STATE_FIELDS + ["im", "hx", "hy", "hz", "shape"]


@dataclass
class Report:
    """BoxStepper.Report (core/box/BoxStepper.java:40) of the last step, with totals over the call."""
    touching: int
    points: int
    rounds: int
    unplaced: int
    unlisted: int
    most_rounds: int = 0
    unplaced_total: int = 0
    unlisted_total: int = 0
    steps: int = 0

    def __iter__(self):
        return iter((self.touching, self.points, self.rounds, self.unplaced, self.unlisted))


def make_params(h, gx, gy, gz, sx, sy, sz, mu_static=0.0, mu_kinetic=0.0, margin=0.0, mu_rolling=0.0):
    """Boxes.params through the library (the same words as vxr.boxes.params)."""
    out = np.zeros(18, dtype=np.int32)
    rc = lib().vxr_box_make_params(h, gx, gy, gz, sx, sy, sz, mu_static, mu_kinetic, margin, mu_rolling, ptr(out))
    if rc:
        raise VxrError(rc, "bad parameters")
    return out


class BoxSimulation:
    """A box/mixed world on one GPU: BoxStep's shape plus BoxSimulation's calls."""

    def __init__(self, bodies: int, substeps: int, sweeps: int = B.WALL_PASSES, symmetric: bool = False,
                 grid: B.Grid | None = None, reach_cells: int = 0, max_pairs: int = 0, device: int = 0,
                 schedule: int = 0, solve_blocks_per_sm: int = 0, _handle=None):
        if _handle is not None:  # made by BatchSimulation
            self.L = lib()
            self.h = _handle
            self.n, self.substeps, self.sweeps, self.grid = bodies, substeps, sweeps, grid
            self._last = Report(0, 0, 0, 0, 0)
            return
        if bodies < 1 or substeps < 1 or sweeps < 1:
            raise ValueError(f"a step needs bodies, substeps and sweeps, got {bodies}, {substeps} and {sweeps}")
        self.L = lib()
        cfg = BoxConfig()
        cfg.bodies, cfg.substeps, cfg.sweeps, cfg.symmetric = bodies, substeps, sweeps, int(bool(symmetric))
        if grid is not None:
            cfg.grid = Grid(grid.nx, grid.ny, grid.nz, grid.cell)
        cfg.reach_cells = reach_cells
        cfg.max_pairs = max_pairs
        cfg.device = device
        cfg.schedule = schedule
        cfg.solve_blocks_per_sm = solve_blocks_per_sm
        status = ctypes.c_int32(0)
        self.h = self.L.vxr_box_create(ctypes.byref(cfg), ctypes.byref(status))
        if not self.h:
            raise VxrError(status.value, "vxr_box_create failed")
        self.n = bodies
        self.substeps = substeps
        self.sweeps = sweeps
        self.grid = grid
        self._last = Report(0, 0, 0, 0, 0)

    # --- the reference's calls ---------------------------------------------------------------------------------

    def start(self, x, y, z, u, v, w, spin, q, half, shape, im, params):
        """BoxSimulation.start: angular velocities in, angular momentum kept."""
        f = [np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z, u, v, w)]
        sp = [np.ascontiguousarray(a, dtype=np.float32) for a in spin]
        qq = [np.ascontiguousarray(a, dtype=np.float32) for a in q]
        hh = [np.ascontiguousarray(a, dtype=np.float32) for a in half]
        sh = np.ascontiguousarray(shape, dtype=np.float32)
        mm = np.ascontiguousarray(im, dtype=np.float32)
        pb = np.ascontiguousarray(params, dtype=np.int32)
        rc = self.L.vxr_box_start(self.h, *[ptr(a) for a in f], ptr_array(sp), ptr_array(qq), ptr_array(hh),
                                  ptr(sh), ptr(mm), ptr(pb))
        self._check(rc)

    def start_momentum(self, x, y, z, u, v, w, l, q, half, shape, im, params):
        """Starts from a state with angular momentum given directly (the test fixture's way)."""
        arrays = [x, y, z, u, v, w, l[0], l[1], l[2], q[0], q[1], q[2], q[3], im, half[0], half[1], half[2], shape]
        f = [np.ascontiguousarray(a, dtype=np.float32) for a in arrays]
        for a in f:
            if a.shape != (self.n,):
                raise ValueError(f"every field holds {self.n} floats")
        pb = np.ascontiguousarray(params, dtype=np.int32)
        self._check(self.L.vxr_box_load_state(self.h, ptr_array(f), ptr(pb)))

    def load_state(self, fields18, params=None):
        """Starts from the 18 fields x y z u v w lx ly lz qx qy qz qw im hx hy hz shape; params None keeps the
        world's (a batch takes its scenes' words with BatchSimulation.scene_params)."""
        f = [np.ascontiguousarray(a, dtype=np.float32) for a in fields18]
        for a in f:
            if a.shape != (self.n,):
                raise ValueError(f"every field holds {self.n} floats")
        pb = None if params is None else np.ascontiguousarray(params, dtype=np.int32)
        self._check(self.L.vxr_box_load_state(self.h, ptr_array(f), ptr(pb)))

    def params(self, params):
        pb = np.ascontiguousarray(params, dtype=np.int32)
        self._check(self.L.vxr_box_params(self.h, ptr(pb)))

    def step_and_wait(self, steps: int = 1) -> Report:
        rep = BoxReport()
        rc = self.L.vxr_box_step(self.h, steps, ctypes.byref(rep))
        self._check(rc)
        self._last = Report(rep.touching, rep.points, rep.rounds, rep.unplaced, rep.unlisted, rep.most_rounds,
                            rep.unplaced_total, rep.unlisted_total, rep.steps)
        return self._last

    def step(self, steps: int = 1) -> Report:
        return self.step_and_wait(steps)

    def gpu_diagnostics(self) -> dict:
        """Diagnostics computed on the GPU (vxr_box_diagnostics): energies, momenta, the deepest contact and wall
        penetration, the fastest speed, non-finite state."""
        d = Diag()
        self._check(self.L.vxr_box_diagnostics(self.h, ctypes.byref(d)))
        return {"kinetic": d.kinetic, "rotational": d.rotational, "potential": d.potential,
                "momentum": tuple(d.momentum), "angular": tuple(d.angular), "max_penetration": d.max_penetration,
                "max_wall_penetration": d.max_wall, "max_speed": d.max_speed, "broken": bool(d.broken)}

    def learned(self, net, mode: int) -> None:
        """The learned warm start: mode 0 off, 1 gather features and targets, 2 start every point from `net`'s
        impulses, 3 only the points that carried nothing (the others keep their carried impulses)."""
        self._check(self.L.vxr_box_learned(self.h, net.h if net is not None else None, mode))

    def first_substeps(self, count: int, solve_only: bool = False) -> None:
        """A measurement: the following steps run only their first `count` substeps (0: whole steps again); with
        solve_only, the last of them skips its relax sweeps."""
        self._check(self.L.vxr_box_first_substeps(self.h, int(count), 1 if solve_only else 0))

    def learned_given(self, answers, fresh_only: bool = False, whole: bool = False) -> None:
        """The next step starts its contact points from what `answers` (a twin world gathering targets) reached in
        its last step, in place of the carried impulses: the network's two targets a point, or with whole the whole
        impulse records (and the walls' records, unless fresh_only); with fresh_only, only the points that carried
        nothing. What a perfect predictor would give. learned(None, 0) ends it."""
        self._check(self.L.vxr_box_learned_given(self.h, answers.h, 1 if fresh_only else 0, 1 if whole else 0))

    def features(self):
        """The last step's gathered rows: features (rows, 16) and targets (rows, 2)."""
        rows = ctypes.c_int32(0)
        self._check(self.L.vxr_box_features(self.h, None, None, 0, ctypes.byref(rows)))
        f = np.zeros((rows.value, 16), np.float32)
        t = np.zeros((rows.value, 2), np.float32)
        self._check(self.L.vxr_box_features(self.h, ptr(f), ptr(t), rows.value, ctypes.byref(rows)))
        return f, t

    def step_graph(self, pairs: int = 1) -> None:
        """pairs x 2 steps as replays of one captured CUDA graph of two whole steps, not waited for (sync waits)."""
        self._check(self.L.vxr_box_step_graph(self.h, pairs))

    def step_async(self, steps: int = 1):
        self._check(self.L.vxr_box_step_async(self.h, steps))

    def sync(self) -> Report:
        rep = BoxReport()
        self._check(self.L.vxr_box_sync(self.h, ctypes.byref(rep)))
        self._last = Report(rep.touching, rep.points, rep.rounds, rep.unplaced, rep.unlisted, rep.most_rounds,
                            rep.unplaced_total, rep.unlisted_total, rep.steps)
        return self._last

    def last(self) -> Report:
        return self._last

    def state(self, out=None) -> list[np.ndarray]:
        """x y z u v w lx ly lz qx qy qz qw, read back; into `out` (13 float32 arrays of n, e.g. in pinned memory)
        when given."""
        if out is None:
            out = [np.empty(self.n, dtype=np.float32) for _ in STATE_FIELDS]
        elif len(out) != len(STATE_FIELDS) or any(a.dtype != np.float32 or a.shape != (self.n,) or
                                                   not a.flags.c_contiguous for a in out):
            raise ValueError(f"out holds {len(STATE_FIELDS)} contiguous float32 arrays of {self.n}")
        self._check(self.L.vxr_box_state(self.h, ptr_array(out)))
        return out

    def state_async(self, out, slot: int) -> None:
        """The state after the steps enqueued so far, read back into `out` (13 contiguous float32 arrays of n, best
        pinned) without waiting: split into slot 0 or 1 on the device and copied on a stream of its own while the next
        steps run. `out` must stay untouched until state_wait(slot)."""
        if len(out) != len(STATE_FIELDS) or any(a.dtype != np.float32 or a.shape != (self.n,) or
                                                 not a.flags.c_contiguous for a in out):
            raise ValueError(f"out holds {len(STATE_FIELDS)} contiguous float32 arrays of {self.n}")
        self._check(self.L.vxr_box_state_async(self.h, ptr_array(out), int(slot)))

    def state_wait(self, slot: int) -> None:
        """Waits until slot `slot`'s last read-back is in its arrays."""
        self._check(self.L.vxr_box_state_wait(self.h, int(slot)))

    def field(self, name: str) -> np.ndarray:
        return self.state()[STATE_FIELDS.index(name)]

    def read_shown(self) -> np.ndarray:
        out = np.empty(B.SHOWN_STRIDE * self.n, dtype=np.float32)
        self._check(self.L.vxr_box_read_shown(self.h, ptr(out)))
        return out

    shown = read_shown

    @property
    def stream(self) -> int:
        return self.L.vxr_box_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.vxr_box_destroy(self.h)
            self.h = None

    __del__ = close

    # --- inspection, for parity -------------------------------------------------------------------------------

    def touching(self):
        """(first, second, points, manifolds (P, 40), impulses (P, 28)) of the last step's touching pairs."""
        n = self.L.vxr_box_touching(self.h, None, None, None, None, None, 0)
        if n < 0:
            raise VxrError(-n, self.error())
        a = np.zeros(n, np.int32)
        b = np.zeros(n, np.int32)
        c = np.zeros(n, np.int32)
        m = np.zeros((n, 40), np.float32)
        imp = np.zeros((n, 28), np.float32)
        got = self.L.vxr_box_touching(self.h, ptr(a), ptr(b), ptr(c), ptr(m), ptr(imp), n)
        if got < 0:
            raise VxrError(-got, self.error())
        return a, b, c, m, imp

    def touching_pairs(self):
        a, b, c, _, _ = self.touching()
        return [(int(x), int(y), int(z)) for x, y, z in zip(a, b, c)]

    def touching_manifolds(self):
        return list(self.touching()[3])

    def touching_impulses(self):
        return list(self.touching()[4])

    def candidate_pairs(self) -> np.ndarray:
        n = self.L.vxr_box_candidates(self.h, None, 0)
        if n < 0:
            raise VxrError(-n, self.error())
        out = np.zeros(2 * n, np.int32)
        got = self.L.vxr_box_candidates(self.h, ptr(out), n)
        if got < 0:
            raise VxrError(-got, self.error())
        return out.reshape(-1, 2)

    def walls(self):
        lam = np.zeros(48 * self.n, np.float32)
        rub = np.zeros(144 * self.n, np.float32)
        rol = np.zeros(144 * self.n, np.float32)
        self._check(self.L.vxr_box_walls(self.h, ptr(lam), ptr(rub), ptr(rol)))
        return lam, rub, rol

    def colour_waves(self) -> int:
        return self.L.vxr_box_colour_waves(self.h)

    def launches(self) -> int:
        return int(self.L.vxr_box_launches(self.h))

    def profile(self, enable: bool) -> np.ndarray:
        """Turns per-phase timing on or off; returns the milliseconds summed since the last call
        (broad phase, narrow phase with carry, colouring, solve)."""
        out = np.zeros(4, np.float64)
        self._check(self.L.vxr_box_profile(self.h, int(bool(enable)), ptr(out)))
        return out

    def activity(self) -> dict:
        out = np.zeros(4, np.int64)
        self._check(self.L.vxr_box_activity(self.h, ptr(out)))
        return {"touching": int(out[0]), "points": int(out[1]), "bodies_active": int(out[2]),
                "wall_records": int(out[3])}

    def trace(self, enable: bool = True) -> np.ndarray:
        """Turns the solve's phase trace on or off; returns the last traced step's entries as (code, ns) rows."""
        out = np.zeros(1 << 16, np.int64)
        n = self.L.vxr_box_trace(self.h, int(bool(enable)), ptr(out), len(out))
        if n < 0:
            raise VxrError(-n, self.error())
        raw = out[:n].astype(np.uint64)
        return np.stack([(raw >> np.uint64(48)).astype(np.int64),
                         (raw & np.uint64((1 << 48) - 1)).astype(np.int64)], axis=1)

    def measure(self, residual: bool = True, cold_start: bool = False, sweeps: int = 0, tolerance: float = 0.0):
        """Gather each sweep's residual; start pair impulses from zero (no warm start); run `sweeps` sweeps (0: the
        created count); stop a substep's sweeps once the residual is at or below `tolerance` (0: never)."""
        self._check(self.L.vxr_box_measure(self.h, int(bool(residual)), int(bool(cold_start)), int(sweeps),
                                           float(tolerance)))
        self.active_sweeps = sweeps or self.sweeps

    def list_kernel(self, tiled: bool) -> None:
        """The broad phase's list by tiles of cells staged in shared memory (True) or a thread a body walking its 27
        cells (False, the default); the pairs are the same either way."""
        self._check(self.L.vxr_box_list_kernel(self.h, int(bool(tiled))))

    def wait_limit(self, ns: int = 0) -> None:
        """The longest a device-wide wait of a step may last (0: the default of 2 s); past it the step stops with
        VXR_ETIMEOUT."""
        self._check(self.L.vxr_box_wait_limit(self.h, int(ns)))

    def contact_errors(self) -> np.ndarray:
        """The positional complementarity error (m) at every contact point of the last step, from the state at its
        end: max(h max(0, -(vn + max(gap, 0) / h)) within the margin, max(0, -gap))."""
        rows = self.L.vxr_box_contact_errors(self.h, None, 0)
        if rows < 0:
            raise VxrError(-rows, self.error())
        out = np.zeros(max(rows, 1), np.float32)
        got = self.L.vxr_box_contact_errors(self.h, ptr(out), rows)
        if got < 0:
            raise VxrError(-got, self.error())
        out = out[:got]
        return out[out >= 0.0]

    def islands(self, enable: bool = True) -> None:
        """Small components solved by island blocks (the default), or every body through the grid-wide phases; the
        results are the same either way."""
        self._check(self.L.vxr_box_islands(self.h, int(bool(enable))))

    def paths(self) -> dict:
        """How the last step was scheduled: bodies through the grid-wide phases, in small components (island blocks),
        in no placed pair (a thread each), and the island groups."""
        out = np.zeros(5, np.int32)
        self._check(self.L.vxr_box_paths(self.h, ptr(out)))
        return {"grid": int(out[0]), "islands": int(out[1]), "alone": int(out[2]), "groups": int(out[3]),
                "largest": int(out[4])}

    def residuals(self):
        """The last step's per-sweep residuals, shape (substeps, 2 sweeps + 1) (warm, solve..., relax...), and the
        sweeps each half-substep ran, shape (substeps, 2)."""
        count = self.L.vxr_box_residuals(self.h, None, 0, None)
        out = np.zeros(count, np.float32)
        used = np.zeros(2 * self.substeps, np.int32)
        got = self.L.vxr_box_residuals(self.h, ptr(out), count, ptr(used))
        if got < 0:
            raise VxrError(-got, self.error())
        return out.reshape(self.substeps, -1), used.reshape(self.substeps, 2)

    def residual_parts(self):
        """The last step's per-sweep residuals in two parts, the pairs' and the walls', each shaped as residuals()
        gives them (their larger is what residuals() gives)."""
        count = self.L.vxr_box_residual_parts(self.h, None, None, 0)
        pairs = np.zeros(count, np.float32)
        walls = np.zeros(count, np.float32)
        got = self.L.vxr_box_residual_parts(self.h, ptr(pairs), ptr(walls), count)
        if got < 0:
            raise VxrError(-got, self.error())
        return pairs.reshape(self.substeps, -1), walls.reshape(self.substeps, -1)

    def error(self) -> str:
        return self.L.vxr_box_error(self.h).decode() if self.h else ""

    def _check(self, rc):
        if rc:
            raise VxrError(rc, self.error())


def collide_pairs(fields18, param_bits, pairs) -> np.ndarray:
    """The narrow phase alone over a flat pair list, through vxr_collide: 40 words per pair."""
    arrs = [np.ascontiguousarray(f, dtype=np.float32) for f in fields18]
    pb = np.ascontiguousarray(param_bits, dtype=np.int32)
    pr = np.ascontiguousarray(pairs, dtype=np.int32)
    npairs = len(pr) // 2
    out = np.zeros(40 * npairs, dtype=np.float32)
    rc = lib().vxr_collide(len(arrs[0]), ptr_array(arrs), ptr(pb), npairs, ptr(pr), ptr(out))
    if rc:
        raise VxrError(rc, "vxr_collide failed")
    return out


class BatchSimulation(BoxSimulation):
    """Many independent scenes stepped as one world (vxr_box_create_batch): bodies numbered scene after scene, each
    scene with its own grid, gravity, walls and friction. Every BoxSimulation call applies to the whole batch; the
    state arrays hold every scene's bodies in order (``first`` gives each scene's first body)."""

    def __init__(self, bodies_per_scene, grids, substeps: int, sweeps: int, symmetric: bool = False,
                 max_pairs: int = 0, device: int = 0, schedule: int = 0, solve_blocks_per_sm: int = 0):
        counts = np.ascontiguousarray(bodies_per_scene, dtype=np.int32)
        table = (Grid * len(grids))(*[Grid(g.nx, g.ny, g.nz, g.cell) for g in grids])
        cfg = BatchConfig()
        cfg.scenes = len(counts)
        cfg.bodies = counts.ctypes.data
        cfg.grids = ctypes.cast(table, ctypes.c_void_p)
        cfg.substeps, cfg.sweeps, cfg.symmetric = substeps, sweeps, int(bool(symmetric))
        cfg.max_pairs, cfg.device, cfg.schedule, cfg.solve_blocks_per_sm = max_pairs, device, schedule, solve_blocks_per_sm
        status = ctypes.c_int32(0)
        h = lib().vxr_box_create_batch(ctypes.byref(cfg), ctypes.byref(status))
        if not h:
            raise VxrError(status.value, "vxr_box_create_batch failed")
        super().__init__(int(counts.sum()), substeps, sweeps, symmetric, None, _handle=h)
        self.scenes = len(counts)
        first = np.zeros(self.scenes + 1, np.int32)
        lib().vxr_box_scenes(self.h, ptr(first))
        self.first = first

    def scene_params(self, params) -> None:
        """Each scene's 18 words, shape (scenes, 18)."""
        p = np.ascontiguousarray(params, dtype=np.int32).reshape(self.scenes, 18)
        self._check(self.L.vxr_box_scene_params(self.h, ptr(p)))
