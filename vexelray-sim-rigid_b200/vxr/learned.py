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


def rows_in_order(feats) -> np.ndarray:
    """Feature rows as int32 words, sorted: two worlds list a round's pairs in the order their threads reached
    them, so the same points can come in another order."""
    v = np.ascontiguousarray(feats, np.float32).view(np.int32)
    return v[np.lexsort(v.T[::-1])]


NETWORK_STARTS = ("carried", "zero", "network_all", "network_new")
CEILING_STARTS = ("answers_all", "answers_new", "first_all", "first_new", "first_whole_all", "first_whole_new")


def compare_starts(scene: dict, state13, net=None, starts=NETWORK_STARTS, samples: int = 3, lead: int = 2,
                   tolerance: float = 1e-4, cap: int = 64, answer_tolerance: float = 1e-6, answer_cap: int = 256,
                   device: int = 0) -> dict:
    """Solve sweeps a substep needs to reach `tolerance` (at most `cap`) from each start, every start on the same
    step. A twin world is made by loading the state (which clears the carried pairs) and stepping `lead` steps at the
    scene's own sweeps, so every twin's measured step starts from the same state and the same carried impulses. The
    starts: "carried" (the reference's warm start), "zero", the network on every point or on the points that carried
    nothing ("network_all", "network_new", modes 2 and 3), and what a perfect predictor would give: the impulses a
    twin's whole step reaches solved to `answer_tolerance` (at most `answer_cap` sweeps), the targets the network is
    trained on ("answers_all", "answers_new"), or the impulses the solve sweeps of a twin's first substep alone reach
    so solved, with no relax sweeps after them: the start from which that substep's solve needs no sweep, given as
    the network's two targets a point ("first_all", "first_new") or as the whole impulse records, friction direction,
    rolling impulses and the walls' records included ("first_whole_all", "first_whole_new"). The answer twins' features are compared with the measured
    twin's as sorted rows (the answers are matched to the points by touching pair). `samples` steps, each from the
    carried twin's state after the one before. Reports each start's mean solve sweeps a substep, its share of
    substeps that reached the tolerance and its mean by substep within the step (a step's start is applied to its
    first substep, the later substeps start from what the substep before reached), and by substep the sweeps the
    pairs' part and the walls' part of the residual would each have needed alone."""
    from .box_simulation import BoxSimulation
    statics = [scene[k] for k in ("im", "hx", "hy", "hz", "shape")]
    room = max(scene["sweeps"], answer_cap, cap)
    reach = scene.get("reach_cells", 0)

    def world():
        return BoxSimulation(scene["bodies"], scene["substeps"], room, False, scene["grid"], reach, device=device)

    needs_net = any(k.startswith("network") for k in starts)
    if needs_net and net is None:
        raise ValueError("the network's starts need a network")
    b = world()
    a = world() if any(k.startswith("answers") for k in starts) else None
    a1 = world() if any(k.startswith("first") for k in starts) else None
    used = {k: [] for k in starts}
    pairs_alone = {k: [] for k in starts}
    walls_alone = {k: [] for k in starts}
    answered = {"answers": [], "first": []}
    answer_residual = {"answers": [], "first": []}
    aligned, checked = True, False
    state = [np.asarray(f, np.float32) for f in state13]

    def twin(w):
        w.learned(None, 0)
        w.first_substeps(0)
        w.load_state(state + statics, scene["params"])
        w.measure(residual=False, sweeps=scene["sweeps"])
        w.step_and_wait(lead)

    def answer(w, substeps):
        twin(w)
        w.first_substeps(substeps, solve_only=substeps > 0)
        w.learned(None, 1)
        w.measure(residual=True, sweeps=answer_cap, tolerance=answer_tolerance)
        w.step_and_wait(1)
        res, ran = w.residuals()
        k = substeps or scene["substeps"]
        last = [float(res[s, int(ran[s, 0])]) for s in range(k)]  # each substep's last solve sweep's residual
        w.first_substeps(0)
        return [int(u) < answer_cap for u in ran[:k, 0]], last, w.features()[0]

    def alone(part, ran):
        """Solve sweeps each substep's part of the residual needed alone: the first within the tolerance."""
        out = []
        for s in range(part.shape[0]):
            n = int(ran[s])
            hit = np.nonzero(part[s, 1:n + 1] <= tolerance)[0]
            out.append(float(hit[0] + 1) if len(hit) else float(n))
        return out

    try:
        for _ in range(samples):
            feats = []
            if a is not None:
                got, last, f = answer(a, 0)
                answered["answers"].extend(got)
                answer_residual["answers"].extend(last)
                feats.append(f)
            if a1 is not None:
                got, last, f = answer(a1, 1)
                answered["first"].extend(got)
                answer_residual["first"].extend(last)
                feats.append(f)
            nxt = None
            for name in starts:
                twin(b)
                if name == "network_all":
                    b.learned(net, 2)
                elif name == "network_new":
                    b.learned(net, 3)
                elif name.startswith("answers"):
                    b.learned_given(a, fresh_only=name.endswith("_new"))
                elif name.startswith("first"):
                    b.learned_given(a1, fresh_only=name.endswith("_new"), whole="whole" in name)
                elif feats:
                    b.learned(None, 1)  # features only: the step is the carried (or zero) start's own
                b.measure(residual=True, cold_start=name == "zero", sweeps=cap, tolerance=tolerance)
                b.step_and_wait(1)
                ran = b.residuals()[1][:, 0]
                used[name].append(ran.astype(np.float64))
                pr, wr = b.residual_parts()
                pairs_alone[name].append(alone(pr, ran))
                walls_alone[name].append(alone(wr, ran))
                if name == "carried":
                    nxt = b.state()
                    if feats:
                        checked = True
                        mine = rows_in_order(b.features()[0])
                        aligned = aligned and all(np.array_equal(mine, rows_in_order(f)) for f in feats)
            b.learned(None, 0)
            state = nxt if nxt is not None else b.state()
    finally:
        for w in (a, a1, b):
            if w is not None:
                w.close()
    mean = {k: float(np.mean(np.concatenate(v))) for k, v in used.items()}
    out = {"samples": samples, "lead_steps": lead, "tolerance_m": tolerance, "cap": cap,
           "mean_sweeps": mean,
           "reached": {k: float(np.mean(np.concatenate(v) < cap)) for k, v in used.items()},
           "by_substep": {k: [float(x) for x in np.mean(np.stack(v), 0)] for k, v in used.items()},
           "pairs_alone_by_substep": {k: [float(x) for x in np.mean(np.array(v), 0)] for k, v in pairs_alone.items()},
           "walls_alone_by_substep": {k: [float(x) for x in np.mean(np.array(v), 0)] for k, v in walls_alone.items()}}
    if "carried" in mean:
        out["gain_vs_carried"] = {k: (mean["carried"] / m if m > 0 else None) for k, m in mean.items()}
    if a is not None or a1 is not None:
        def worst(v):
            return {"median": float(np.median(v)), "max": float(np.max(v))} if v else None
        out["answers"] = {"tolerance_m": answer_tolerance, "cap": answer_cap,
                          "reached_whole_step": float(np.mean(answered["answers"])) if answered["answers"] else None,
                          "reached_first_substep": float(np.mean(answered["first"])) if answered["first"] else None,
                          "last_solve_residual_m": {"whole_step": worst(answer_residual["answers"]),
                                                    "first_substep": worst(answer_residual["first"])}}
        out["twins_aligned"] = bool(aligned) if checked else None
    return out


def judge(scene: dict, state13, net, samples: int = 3, tolerance: float = 1e-4, cap: int = 64, ceiling: bool = False,
          device: int = 0) -> dict:
    """The plain solver judges the network, every start on the same steps (compare_starts from `state13`): sweeps to
    the residual from the network's impulses on every point (mode 2) and on the points that carried nothing (mode 3),
    against from the carried ones and from zero. The network is kept, in its better mode, only if it needs fewer
    sweeps than the carried impulses; otherwise the plain warm start is the fallback. With `ceiling`, the same steps
    are also taken from the answers a perfect predictor would give."""
    starts = NETWORK_STARTS + (CEILING_STARTS if ceiling else ())
    r = compare_starts(scene, state13, net, starts=starts, samples=samples, tolerance=tolerance, cap=cap,
                       device=device)
    m, reached = r["mean_sweeps"], r["reached"]
    plain, cold, learned, fresh = m["carried"], m["zero"], m["network_all"], m["network_new"]
    best_mode, best = (2, learned) if learned <= fresh else (3, fresh)
    use = best < plain
    verdict = {"plain_warm_start": plain, "plain_warm_start_reached": reached["carried"], "plain_cold_start": cold,
               "plain_cold_start_reached": reached["zero"], "learned": learned,
               "learned_reached": reached["network_all"], "learned_new_contacts_only": fresh,
               "learned_new_contacts_only_reached": reached["network_new"],
               "gain_vs_warm_start": plain / best if best > 0 else None,
               "gain_vs_cold_start": cold / best if best > 0 else None,
               "kept": bool(use), "mode": best_mode if use else 0,
               "fallback": None if use else "plain warm start (the network needs no fewer sweeps in either mode)",
               "same_steps": {"samples": samples, "lead_steps": r["lead_steps"], "by_substep": r["by_substep"],
                              "pairs_alone_by_substep": r["pairs_alone_by_substep"],
                              "walls_alone_by_substep": r["walls_alone_by_substep"]}}
    if ceiling:
        verdict["ceiling"] = {"mean_sweeps": {k: m[k] for k in CEILING_STARTS},
                              "reached": {k: reached[k] for k in CEILING_STARTS},
                              "gain_vs_carried": {k: r["gain_vs_carried"][k] for k in CEILING_STARTS},
                              "answers": r["answers"], "twins_aligned": r["twins_aligned"]}
    return verdict
