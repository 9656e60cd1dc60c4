"""The learned warm start's network (include/vxr.h, vxr_mlp_*): a 16 -> 64 -> 64 -> 2 SiLU multilayer perceptron
with BF16 weights and FP32 accumulation, run and trained on the GPU by the library's tensor-core kernels. No reference
counterpart: the reference warm-starts a contact with the impulses it took last step (core/box/BoxPairs.java:191-267).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import VxrError, lib, ptr

IN, HID, OUT = 16, 64, 2
PARAMS = 5378
LAYOUT = [("w1", (IN, HID)), ("b1", (HID,)), ("w2", (HID, HID)), ("b2", (HID,)), ("w3", (HID, OUT)), ("b3", (OUT,))]


def unpack(flat) -> dict:
    out, at = {}, 0
    for name, shape in LAYOUT:
        size = int(np.prod(shape))
        out[name] = np.asarray(flat[at:at + size], dtype=np.float32).reshape(shape)
        at += size
    return out


def pack(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[name], np.float32).reshape(-1) for name, _ in LAYOUT])


class Mlp:
    def __init__(self, device: int = 0, seed: int = 0):
        status = ctypes.c_int32(0)
        self.h = lib().vxr_mlp_create(device, seed, ctypes.byref(status))
        if not self.h:
            raise VxrError(status.value, "vxr_mlp_create")

    def _check(self, rc):
        if rc != 0:
            raise VxrError(rc, lib().vxr_mlp_error(self.h).decode())

    def set(self, params=None, mean=None, inv_std=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in
                (pack(params) if isinstance(params, dict) else params, mean, inv_std)]
        self._check(lib().vxr_mlp_set(self.h, *[ptr(a) for a in arrs]))

    def get(self):
        p = np.zeros(PARAMS, np.float32)
        m = np.zeros(IN, np.float32)
        s = np.zeros(IN, np.float32)
        self._check(lib().vxr_mlp_get(self.h, ptr(p), ptr(m), ptr(s)))
        return unpack(p), m, s

    def forward(self, features) -> np.ndarray:
        f = np.ascontiguousarray(features, np.float32)
        out = np.zeros((f.shape[0], OUT), np.float32)
        self._check(lib().vxr_mlp_forward(self.h, ptr(f), f.shape[0], ptr(out)))
        return out

    def gradients(self, features, targets):
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        g = np.zeros(PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(lib().vxr_mlp_gradients(self.h, ptr(f), ptr(t), f.shape[0], ptr(g), ptr(loss)))
        return unpack(g), float(loss[0])

    def train(self, features, targets, epochs=20, batch=4096, lr=1e-3, seed=0) -> np.ndarray:
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(lib().vxr_mlp_train(self.h, ptr(f), ptr(t), f.shape[0], epochs, batch, lr, seed, ptr(losses)))
        return losses[:epochs]

    def close(self):
        if getattr(self, "h", None):
            lib().vxr_mlp_destroy(self.h)
            self.h = None

    __del__ = close


# --- the workflow: gather, train, judge ----------------------------------------------------------------------------

def settled_world(scene: dict, settle: int, sweeps_cap: int, device: int = 0):
    """A box world of `scene` (room for `sweeps_cap` sweeps a half-substep), stepped `settle` steps with the scene's
    own sweeps."""
    from .box_simulation import BoxSimulation
    w = BoxSimulation(scene["bodies"], scene["substeps"], max(scene["sweeps"], sweeps_cap), False, scene["grid"],
                      device=device)
    w.measure(residual=False, sweeps=scene["sweeps"])
    w.start_momentum(scene["x"], scene["y"], scene["z"], scene["u"], scene["v"], scene["w"],
                     [scene["lx"], scene["ly"], scene["lz"]], [scene["qx"], scene["qy"], scene["qz"], scene["qw"]],
                     [scene["hx"], scene["hy"], scene["hz"]], scene["shape"], scene["im"], scene["params"])
    if settle:
        w.step_and_wait(settle)
    return w


def gather(world, steps: int, rows_wanted: int, sweeps_cap: int = 64, tolerance: float = 1e-6):
    """Training rows from the plain solver run to `tolerance` (at most `sweeps_cap` sweeps a half-substep): each
    step's contact points, their features at the step's start and the impulses its solve reached."""
    world.learned(None, 1)
    world.measure(residual=True, sweeps=sweeps_cap, tolerance=tolerance)
    feats, targets = [], []
    have = 0
    for _ in range(steps):
        world.step_and_wait(1)
        f, t = world.features()
        feats.append(f)
        targets.append(t)
        have += len(f)
        if have >= rows_wanted:
            break
    world.learned(None, 0)
    f = np.concatenate(feats)[:rows_wanted]
    t = np.concatenate(targets)[:rows_wanted]
    return f, t


def gather_many(plan, rows_wanted: int, sweeps_cap: int = 64, tolerance: float = 1e-6, device: int = 0):
    """Training rows from several worlds and phases of the drop: `plan` lists (scene, steps to settle first); each
    entry gives an equal share of `rows_wanted`, from as many steps as that takes (the plain solver run to `tolerance`,
    at most `sweeps_cap` sweeps a half-substep). Returns the features, the targets and each row's plan entry."""
    share = max(1, rows_wanted // max(len(plan), 1))
    feats, targets, source = [], [], []
    for k, (scene, settle) in enumerate(plan):
        w = settled_world(scene, settle, sweeps_cap, device=device)
        f, t = gather(w, steps=64, rows_wanted=share, sweeps_cap=sweeps_cap, tolerance=tolerance)
        w.close()
        feats.append(f)
        targets.append(t)
        source.append(np.full(len(f), k, np.int32))
    return np.concatenate(feats), np.concatenate(targets), np.concatenate(source)


def new_contacts(feats) -> np.ndarray:
    """The rows of points that carried nothing from the step before (features 7 and 8, the carried impulses, zero):
    where the reference's start is zero, and where the network's start replaces it (mode 3)."""
    f = np.asarray(feats, np.float32)
    return (f[:, 7] == 0.0) & (f[:, 8] == 0.0)


def prediction_errors(net, feats, targets) -> dict:
    """How close each start is to the impulses the plain solver reaches (both scaled by the pair's effective mass
    x |g| x h, as the features and targets are): the network's (its outputs, negatives clipped to zero, as the step
    applies them) against the carried impulses (features 7 and 8) on the points that carried something, and against
    zero on those that carried nothing. Root mean square over the rows, normal and tangential together."""
    f = np.asarray(feats, np.float32)
    t = np.asarray(targets, np.float32)
    pred = np.maximum(net.forward(f), 0.0)
    carried = (f[:, 7] != 0.0) | (f[:, 8] != 0.0)
    rms = lambda a, b: float(np.sqrt(np.mean(np.sum((a - b) ** 2, 1)))) if len(a) else None  # noqa: E731
    return {"rows": int(len(f)), "carried_rows": int(carried.sum()),
            "carried": {"network": rms(pred[carried], t[carried]), "carried_impulses": rms(f[carried][:, 7:9],
                                                                                             t[carried])},
            "new": {"network": rms(pred[~carried], t[~carried]),
                    "zero": rms(np.zeros_like(t[~carried]), t[~carried])}}


def sweeps_to_residual(world, steps: int, tolerance: float, cap: int, mode: int, net=None, cold: bool = False):
    """Mean solve sweeps a substep takes to reach the residual (at most `cap`), over `steps` steps, and the share of
    substeps that reached it: the plain warm start (mode 0, or cold = from zero) or the network's (mode 2 or 3)."""
    world.learned(net, mode)
    world.measure(residual=True, cold_start=cold, sweeps=cap, tolerance=tolerance)
    used_all = []
    for _ in range(steps):
        world.step_and_wait(1)
        _, used = world.residuals()
        used_all.extend(int(u) for u in used[:, 0])
    world.learned(None, 0)
    return float(np.mean(used_all)), float(np.mean([u < cap for u in used_all]))


def judge(world, net, steps: int = 3, tolerance: float = 1e-4, cap: int = 64) -> dict:
    """The plain solver judges the network: sweeps to the residual from its impulses against from the carried ones
    (and from zero), each over the same number of steps from where the world is. The network is tried on every
    point (mode 2) and on the points that carried nothing (mode 3, the carried impulses kept elsewhere). It is kept,
    in its better mode, only if it needs fewer sweeps; otherwise the plain warm start is the fallback."""
    plain, plain_reached = sweeps_to_residual(world, steps, tolerance, cap, 0)
    cold, cold_reached = sweeps_to_residual(world, steps, tolerance, cap, 0, cold=True)
    learned, learned_reached = sweeps_to_residual(world, steps, tolerance, cap, 2, net)
    fresh, fresh_reached = sweeps_to_residual(world, steps, tolerance, cap, 3, net)
    best_mode, best = (2, learned) if learned <= fresh else (3, fresh)
    use = best < plain
    return {"plain_warm_start": plain, "plain_warm_start_reached": plain_reached, "plain_cold_start": cold,
            "plain_cold_start_reached": cold_reached, "learned": learned, "learned_reached": learned_reached,
            "learned_new_contacts_only": fresh, "learned_new_contacts_only_reached": fresh_reached,
            "gain_vs_warm_start": plain / best if best > 0 else None,
            "gain_vs_cold_start": cold / best if best > 0 else None,
            "kept": bool(use), "mode": best_mode if use else 0,
            "fallback": None if use else "plain warm start (the network needs no fewer sweeps in either mode)"}
