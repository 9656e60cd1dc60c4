"""The autotuner for batched scenes: which cell size, solve block shape and schedule of the coloured rounds step a
batch fastest on this GPU. No reference counterpart (the reference fixes its cell by BoxBroad.grid's rule,
core/box/BoxBroad.java:66-68, and runs its rounds one dispatch after another, core/box/BoxStep.java:217-231).

The schedule of the rounds has two knobs: whether the small connected components of the placed pairs are solved
whole by one warp each (islands) or go through the grid-wide phases with the rest, and whether the grid-wide phases
run each round behind a grid barrier or as a stream of items each waiting for its own bodies (dependency).

The search is timed, not modelled: the batch is stepped once to a representative state (bodies landed and piling),
then every candidate steps from that same state, a few steps to warm the pair impulses and a few timed with CUDA
events, and the fastest wins. The result is cached per GPU model and batch shape (a JSON file under
$VXR_TUNE_CACHE, default ~/.cache/vxr-b200/tune.json), so a second run of the same shape does not search again.

The candidates cannot change a result, only its speed: every cell size is at least the reference's rule (the
27-cell neighbourhood still holds every pair), and both schedules and every block shape keep each body's order of
operations. (The one exception, stated for completeness: a body with more than 32 partners keeps the first 32 the
neighbourhood walk finds, and cell size changes the walk's order.) The colouring itself is the reference's greedy
one in every candidate: its rounds are the reference's, so they are not a knob.
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time

import numpy as np

from . import boxes as B

CELL_SCALES = (1.0, 1.25)
BLOCKS_PER_SM = (1, 2)
SCHEDULES = (0, 1)
ISLANDS = (True, False)


def candidates():
    """Every (cell scale, solve blocks an SM, grid schedule, islands) the search times."""
    return list(itertools.product(CELL_SCALES, BLOCKS_PER_SM, SCHEDULES, ISLANDS))


def cache_path() -> str:
    return os.environ.get("VXR_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "vxr-b200", "tune.json"))


def _key(batch: dict, device_name: str) -> str:
    c = np.asarray(batch["counts"])
    return (f"{device_name}|scenes={len(c)}|bodies={int(c.sum())}|substeps={batch['substeps']}|"
            f"sweeps={batch['sweeps']}")


def scaled_grids(batch: dict, scale: float):
    """Each scene's grid with cells `scale` times the rule's side (never below it)."""
    out = []
    for g, (sx, sy, sz) in zip(batch["grids"], batch["walls"]):
        cell = g.cell * max(1.0, scale)
        out.append(B.Grid(max(1, math.ceil(sx / cell)), max(1, math.ceil(sy / cell)), max(1, math.ceil(sz / cell)),
                          float(np.float32(cell))))
    return out


def _fields(batch: dict, state=None):
    from . import scenes
    f = [batch[k] for k in scenes.FIELDS]
    if state is not None:
        f[:13] = state
    return f


def make_batch(batch: dict, cand, state=None, device: int = 0):
    """A batched world of `batch` set up as candidate `cand` (cell scale, solve blocks an SM, grid schedule,
    islands), from the batch's start or from `state` (its 13 moving fields)."""
    from .box_simulation import BatchSimulation
    scale, per_sm, schedule, islands = cand
    sim = BatchSimulation(batch["counts"], scaled_grids(batch, scale), batch["substeps"], batch["sweeps"],
                          device=device, schedule=schedule, solve_blocks_per_sm=per_sm)
    sim.load_state(_fields(batch, state), None)
    sim.scene_params(batch["params"])
    sim.islands(islands)
    return sim


def tune_batch(batch: dict, device: int = 0, settle_steps: int = 120, warm_steps: int = 4, timed_steps: int = 6,
               use_cache: bool = True, verbose: bool = False) -> dict:
    """The fastest of CELL_SCALES x BLOCKS_PER_SM x SCHEDULES for this batch on this GPU (cached)."""
    import torch
    name = torch.cuda.get_device_name(device)
    key = _key(batch, name)
    path = cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                cache = json.load(f)
        except Exception:
            cache = {}
        if key in cache:
            return dict(cache[key], cached=True)

    # a representative state: the batch stepped until its bodies have landed
    sim = make_batch(batch, (1.0, 0, 0, True), None, device)
    sim.step_and_wait(settle_steps)
    state = sim.state()
    sim.close()
    trials = []
    for cand in candidates():
        scale, per_sm, schedule, islands = cand
        sim = make_batch(batch, cand, state, device)
        sim.step_and_wait(warm_steps)
        stream = torch.cuda.ExternalStream(sim.stream)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        sim.step_async(timed_steps)
        end.record(stream)
        sim.sync()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end) / timed_steps
        sim.close()
        trials.append({"cell_scale": scale, "solve_blocks_per_sm": per_sm, "schedule": schedule, "islands": islands,
                       "ms_per_step": ms})
        if verbose:
            print(trials[-1])
    best = min(trials, key=lambda t: t["ms_per_step"])
    result = {"cell_scale": best["cell_scale"], "solve_blocks_per_sm": best["solve_blocks_per_sm"],
              "schedule": best["schedule"], "islands": best["islands"], "ms_per_step": best["ms_per_step"],
              "trials": trials,
              "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    if use_cache:
        cache[key] = result
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    return dict(result, cached=False)
