"""Benchmark: body-steps/s of the box/mixed rigid-body step on the large mixed scene (262,144 bodies).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vxr|reference]

One "step" is one simulation step of the scene: broad phase, narrow phase, warm-start carry, colouring and four
substeps of ten sweeps of the coloured soft-step solve, all on the GPU. The scene is the large mixed configuration
(seeded synthetic bodies of its shapes, sizes and distributions). The timed steps are steps W..W+K-1 of the drop.

value : body-steps/s with the state resident in HBM, each step timed with CUDA events on the world's stream, L2
        flushed (a 256 MiB write) before every timed step, summed over the K steps; max over ranks.
e2e   : the same metric through the C-ABI with host buffers: each step new parameters copied in, one
        vxr_box_step, and the state (13 floats a body) read back to host memory; wall clock, max over ranks.
roofline : the solve kernel (the dominant one), algorithmic bytes per launch from the activity counted in the run
        over its CUDA-event time, against the measured HBM copy bandwidth.
cpu_baseline : the CPU oracle (a C++ restatement of the reference's kernels; the reference itself is Java built
        on a library absent from this machine) with OpenMP on every host core, on a 1/16-volume sample of the scene.

With N > 1 GPUs the scene does not shard (one connected pile): each rank steps its own replica (a different seed),
and value sums the ranks' body-steps over the slowest rank's time ("replicas only").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "vexelray-sim-rigid_b200"))
sys.path.insert(0, ROOT)

METRIC = "body-steps/s on 1 B200; solver iters to residual≤1e-4 m, warm-start vs plain"
UNIT = "body-steps/s"
BODIES = 262_144


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clocks and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, every_ms: int = 50):
        self.device = device
        self.every_ms = every_ms
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.every_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 8 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 8 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, name in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


class Reports:
    """The step reports of a timed loop, gathered over its periodic syncs. vxr_box_sync hands over the totals of the
    steps since the sync before and zeroes them, so a sync with no step since reports nothing: the last step's
    counts are kept from the last sync that covered a step, and the totals summed over all of them."""

    def __init__(self):
        self.last = None
        self.unplaced_total = 0
        self.unlisted_total = 0
        self.most_rounds = 0
        self.steps = 0

    def add(self, rep):
        if rep.steps > 0:
            self.last = rep
            self.unplaced_total += int(rep.unplaced_total)
            self.unlisted_total += int(rep.unlisted_total)
            self.most_rounds = max(self.most_rounds, int(rep.most_rounds))
            self.steps += int(rep.steps)
        return rep

    def finish(self, world, synced_every: int, steps: int):
        """The final sync, made only where steps ran since the loop's last periodic one."""
        if steps % synced_every or self.last is None:
            self.add(world.sync())
        return self

    def last_step(self) -> dict:
        r = self.last
        if r is None:
            return {"touching": 0, "points": 0, "rounds": 0, "unplaced": 0, "unlisted": 0}
        return {"touching": int(r.touching), "points": int(r.points), "rounds": int(r.rounds),
                "unplaced": int(r.unplaced), "unlisted": int(r.unlisted), "most_rounds": self.most_rounds,
                "unplaced_total": self.unplaced_total, "unlisted_total": self.unlisted_total,
                "steps_reported": self.steps}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def _reduce(pg, value: float, op) -> float:
    import torch
    device = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=op)
    return float(t.item())


def all_max(pg, value: float) -> float:
    """The largest of the ranks' values (a time: the job is as slow as its slowest rank)."""
    return value if pg is None else _reduce(pg, value, pg.ReduceOp.MAX)


def all_sum(pg, value: float) -> float:
    return value if pg is None else _reduce(pg, value, pg.ReduceOp.SUM)


def whole_job_rate(pg, units: float, steps: int, ms: float) -> float:
    """Units all ranks stepped, per second of the slowest rank's device time: this rank stepped `units` bodies
    `steps` times in `ms` milliseconds."""
    return all_sum(pg, float(units)) * steps / (all_max(pg, ms) / 1e3)


def shard_scenes(scenes: int, world_size: int, rank: int) -> list:
    """This rank's scenes of a batch: scene k to rank k mod N. No data-path collective: the scenes are
    independent."""
    return [k for k in range(scenes) if k % world_size == rank]


def barrier(pg):
    if pg is not None:
        pg.barrier()


ITERATION_CAP = 64


# The landed-pile window's first step: by then the bodies from the top of the 64 m volume have landed (a drop of 64 m
# takes about 3.6 s, 430 steps of 1/120 s).
LANDED_STEP = 480
# DRAM traffic of the solve's launches, each from an ncu capture of one launch with one pass (dram__bytes_read.sum +
# dram__bytes_write.sum). In the timed window (step 5 of the default run) every component fits a block, so the solve
# is the island kernel and the grid kernel exits at once: its traffic is the island kernel's. Late in the drop (the
# step after 480, the state saved at step 480 and loaded) one pile holds nearly every body and the grid kernel does
# the solve; there the pair records outgrow L2. Each launch's own algorithmic bytes are given beside it.
EARLY_SOLVE_TRAFFIC = {"step": 5, "kernel": "k_islands", "dram_bytes": 45.11e6, "dram_read_bytes": 41.78e6,
                       "dram_write_bytes": 3.33e6, "algorithmic_bytes": 1.72e9, "ms": 5.87,
                       "source": "ncu, one launch, one pass"}
LATE_SOLVE_TRAFFIC = {"step": 481, "kernel": "k_solve", "dram_bytes": 5.17e9, "dram_read_bytes": 3.76e9,
                      "dram_write_bytes": 1.41e9, "algorithmic_bytes": 7.85e9, "ms": 18.85, "source": "ncu, one launch"}


def make_world(scene, device, max_pairs=0, schedule=0, solve_blocks_per_sm=0, islands=True):
    from vxr.box_simulation import BoxSimulation
    # room for the iteration count measurement's sweeps; the steps run the scene's own
    w = BoxSimulation(scene["bodies"], scene["substeps"], max(scene["sweeps"], ITERATION_CAP), False, scene["grid"],
                      reach_cells=scene.get("reach_cells", 1), device=device, max_pairs=max_pairs, schedule=schedule,
                      solve_blocks_per_sm=solve_blocks_per_sm)
    w.measure(residual=False, sweeps=scene["sweeps"])
    w.islands(islands)
    l = [scene["lx"], scene["ly"], scene["lz"]]
    q = [scene["qx"], scene["qy"], scene["qz"], scene["qw"]]
    h = [scene["hx"], scene["hy"], scene["hz"]]
    w.start_momentum(scene["x"], scene["y"], scene["z"], scene["u"], scene["v"], scene["w"], l, q, h,
                     scene["shape"], scene["im"], scene["params"])
    return w


def with_cell(scene, cell):
    """The scene on a grid of `cell`-wide cells; where that is narrower than the reference's rule (BoxBroad.grid),
    the neighbourhood walk widens to as many cells each way as the rule's cell spans."""
    from vxr import boxes as B
    sx, sy, sz = scene["walls"]
    rule = scene["grid"].cell
    scene["grid"] = B.covering(sx, sy, sz, cell)
    scene["reach_cells"] = max(1, math.ceil(rule / scene["grid"].cell))
    return scene


def window_quality(w, scene, steps):
    """What `steps` more steps of `w` leave behind, at the scene's own sweep count: each substep's residual after
    its last solve sweep and after its last relax sweep (the largest positional correction that sweep still made,
    h k (|dlambda_n| + |dlambda_t|)), and each contact point's complementarity error at the step's end (the larger of
    h max(0, -(vn + max(gap, 0) / h)) within the margin and the overlap max(0, -gap)). Measuring changes no result."""
    sweeps = scene["sweeps"]
    w.measure(residual=True, sweeps=sweeps)
    solve_res, relax_res, errs_max, errs_p99, points = [], [], [], [], 0
    for _ in range(steps):
        w.step_and_wait(1)
        res, _ = w.residuals()
        solve_res.extend(res[:, sweeps].tolist())
        relax_res.extend(res[:, 2 * sweeps].tolist())
        e = w.contact_errors()
        points += len(e)
        if len(e):
            errs_max.append(float(e.max()))
            errs_p99.append(float(np.percentile(e, 99)))
    w.measure(residual=False, sweeps=sweeps)
    s, r = np.array(solve_res), np.array(relax_res)
    return {"steps": steps, "sweeps": sweeps,
            "update_residual_m": {"after_last_solve_sweep": {"max": float(s.max()), "p99": float(np.percentile(s, 99)),
                                                             "median": float(np.median(s))},
                                  "after_last_relax_sweep": {"max": float(r.max()), "p99": float(np.percentile(r, 99)),
                                                             "median": float(np.median(r))},
                                  "substeps_at_or_below_1e-4": float(np.mean(s <= 1e-4))},
            "complementarity_m": {"max": max(errs_max) if errs_max else 0.0,
                                  "p99_median_over_steps": float(np.median(errs_p99)) if errs_p99 else 0.0,
                                  "points_per_step": points / max(steps, 1)},
            "definitions": "update residual: a sweep's largest positional correction at any contact point; "
                           "complementarity: per contact point at the step's end, "
                           "max(h max(0, -(vn + max(gap,0)/h)) within the margin, max(0, -gap))"}


def timed_steps(w, stream, flush, steps):
    """`steps` steps of `w`, each timed with CUDA events on the world's stream, L2 flushed before each."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            starts[k].record(stream)
        w.step_async(1)
        with torch.cuda.stream(stream):
            ends[k].record(stream)
    w.sync()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in zip(starts, ends)]


def algorithmic_solve_bytes(n, substeps, sweeps, touching, points, active, wall_records):
    """Bytes one solve launch (a step's substeps) must move: S [124 N + (2I+1)(96 N_c + P (16 + 88 k) + 56 W)],
    P touching pairs, k points per pair, N_c bodies in a contact, W wall contact records held."""
    k = points / touching if touching else 0.0
    per_sweep = 96 * active + touching * (16 + 88 * k) + 56 * wall_records
    return substeps * (124 * n + (2 * sweeps + 1) * per_sweep)


def cpu_baseline(steps_timed: int = 24, warm: int = 2, fraction: float = 1 / 16):
    """The oracle with OpenMP on every host core, on a 1/16-volume sample of the scene (same density)."""
    from oracle.box import OracleBoxWorld, lib as orc_lib
    from vxr import scenes
    scene = scenes.sub_volume(BODIES, fraction)
    w = OracleBoxWorld(scene["bodies"], scene["substeps"], scene["sweeps"], False, scene["grid"], threads=True)
    for k in scenes.FIELDS:
        w.set_field(k, scene[k])
    w.set_params(scene["params"])
    w.step(warm)
    t0 = time.perf_counter()
    w.step(steps_timed)
    dt = time.perf_counter() - t0
    cores = int(orc_lib(True).orc_threads())
    w.close()
    return {"value": scene["bodies"] * steps_timed / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{scene['bodies']} bodies (1/16 of the volume at the same density), steps {warm}.."
                      f"{warm + steps_timed - 1} of the drop, {dt:.1f} s, OpenMP C++ oracle"}


SPHERE_WORKLOAD = ("sphere lattice: 1,024 spheres r 0.5 m rho 1000 on a 16x8x8 lattice at 1.2 m, jitter U(+-0.05) "
                   "m, at rest, into an open 20x20 m box; dt 1/60 s, 4 substeps, 8 Gauss-Seidel iterations run until "
                   "done, mu 0.5, e 0.2, grid cell 1.0 m")


def sphere_step_bytes(n, substeps, iterations, listed, rounds):
    """Bytes one sphere step must move: per substep, the state (112 B a sphere) read and written by each of the
    per-sphere passes (predict and bin, warm walls, list, velocity, restitution, the walls of every pass); the list
    made (pair, links and 7 impulse words, 48 B a place); per round every open place read (pair and mark, 12 B); and
    per pass and phase every contact solved once (both spheres' state read, 160 B, and written, 96 B, and its
    impulses read and written, 64 B). `rounds` is the step's rounds over every pass (parting; rubbing runs as many)."""
    per_sphere = 224 * (5 + iterations)
    per_substep = n * per_sphere + 48 * listed + 2 * iterations * listed * (160 + 96 + 64)
    return substeps * per_substep + 2 * rounds * listed * 12


def sphere_cpu_baseline(scene, warm, steps):
    """The oracle (serial C++ restatement) on the same scene: steps warm..warm+steps-1, timed on the host."""
    from oracle.sphere import OracleSphereWorld
    from vxr import spheres as S
    w = OracleSphereWorld(scene["spheres"], scene["substeps"], scene["iterations"], S.GAUSS_SEIDEL_BY_CONTACT,
                          scene["grid"])
    for k in ("x", "y", "z", "u", "v", "w", "r", "im"):
        w.set_field(k, scene[k])
    w.set_shown(S.shown_at_start(scene["x"], scene["y"], scene["z"], scene["r"]))
    w.set_params(scene["params"], S.rubs(scene["params"]))
    w.step(warm)
    t0 = time.perf_counter()
    w.step(steps)
    dt = time.perf_counter() - t0
    w.close()
    return {"value": scene["spheres"] * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"the whole scene, steps {warm}..{warm + steps - 1}, {dt:.1f} s, serial C++ oracle"}


def picture_timing(world, shape, n, extent, device, squash=1.5, side=1024, draws=20, cpu=True):
    """The picture of the world's last step (its resident `shown`, where the ring would hand it to a reader),
    side x side pixels from an orbit camera, timed with CUDA events over `draws` draws after 3 untimed ones; every
    pixel tests every body, as the reference's shaders do. The oracle's restatement times a band of rows on one core
    as the CPU figure."""
    import ctypes

    import torch

    from vxr import picture as P
    from vxr._lib import lib
    words = ctypes.c_int64(0)
    if shape == P.SPHERES:
        src = lib().vxr_sphere_shown_device(world._h, ctypes.byref(words))
    else:
        src = lib().vxr_box_shown_device(world.h, ctypes.byref(words))
    # a box with its lid far above is framed as a cube of its footprint
    extent = (extent[0], min(extent[1], max(extent[0], extent[2])), extent[2])
    cam = P.orbit_camera(extent, (1.1, 0.7, -1.5), alpha=0.5, squash=squash)
    rgb = torch.empty((side, side, 3), device=f"cuda:{device}")
    torch.cuda.synchronize()
    for _ in range(3):
        P.draw(shape, src, n, cam, side, side, rgb)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(draws):
        P.draw(shape, src, n, cam, side, side, rgb)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / draws
    tests = side * side * n
    out = {"pixels": [side, side], "bodies": n, "ms_per_picture": ms, "pixels_per_s": side * side / (ms / 1e3),
           "ray_body_tests_per_s": tests / (ms / 1e3), "draws": draws}
    if cpu:
        from oracle import picture as OP
        shown = world.read_shown()
        band = max(1, min(side // 64, int(2e8 // (side * max(n, 1)))))  # about 2e8 bounding tests
        t0 = time.perf_counter()
        OP.picture(shape, shown, P.push_words(cam, n), side, side, rows=range(side // 2, side // 2 + band))
        dt = time.perf_counter() - t0
        out["cpu_oracle"] = {"pixels_per_s": side * band / dt, "cores": 1, "kind": "port",
                             "sample": f"the {band} middle rows of the same picture, {dt:.1f} s"}
    return out


def run_spheres(args):
    """The plain sphere scene on the sphere package: one persistent kernel a step."""
    world_size, rank, local, pg = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from vxr import scenes
    from vxr import spheres as S
    from vxr.sphere_simulation import SphereSimulation
    scene = scenes.sphere_lattice(seed=1 + rank)
    n = scene["spheres"]

    def make():
        sim = SphereSimulation(n, scene["substeps"], scene["iterations"], scene["grid"], S.GAUSS_SEIDEL_BY_CONTACT,
                               device=local, blocks=args.sphere_blocks, cluster=args.sphere_cluster)
        sim.start(scene["x"], scene["y"], scene["z"], scene["u"], scene["v"], scene["w"], scene["r"], scene["im"],
                  scene["params"])
        return sim

    sim = make()
    stream = torch.cuda.ExternalStream(sim.stream())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    sim.step_and_wait(args.warmup)
    launches0 = sim.launches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    rounds, listed = [], []
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            sim.step_async(1)
            with torch.cuda.stream(stream):
                ends[k].record(stream)
            rep = sim.sync()
            rounds.append(rep.rounds)
            listed.append(int(sim.counts()[S.LISTED]))
    torch.cuda.synchronize()
    barrier(pg)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    launches = sim.launches() - launches0
    total_ms = float(sum(step_ms))
    slowest_ms = all_max(pg, total_ms)
    bodies_all = all_sum(pg, float(n))
    value = bodies_all * args.steps / (slowest_ms / 1e3)
    hbm, which = peaks()
    b = [sphere_step_bytes(n, scene["substeps"], scene["iterations"], min(l, 6 * n), r)
         for l, r in zip(listed, rounds)]
    achieved = sum(b) / (total_ms / 1e3) / 1e9
    pic = picture_timing(sim, 0, n, scene["walls"], local, cpu=rank == 0 and not args.no_cpu)
    sim.close()

    e2e = None
    if not args.no_e2e:
        sim2 = make()
        # the step's result read into pinned host arrays, reused every step
        pinned = [torch.empty(n, dtype=torch.float32, pin_memory=True).numpy() for _ in range(9)]
        for _ in range(args.warmup):
            sim2.step_and_wait(1)
            sim2.state(pinned)
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sim2.params(scene["params"])
            sim2.step_and_wait(1)
            sim2.state(pinned)
        e2e_s = all_max(pg, time.perf_counter() - t0)
        sim2.close()
        e2e = {"value": bodies_all * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 13 * 4,
               "d2h_bytes_per_step": 9 * 4 * n}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": slowest_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": SPHERE_WORKLOAD, "spheres": n, "dt": scene["dt"], "substeps": scene["substeps"],
                   "iterations": scene["iterations"], "timed_steps": f"{args.warmup}..{args.warmup + args.steps - 1}",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": "replicas" if world_size > 1 else "single"},
        "rounds_per_step": {"mean": float(np.mean(rounds)), "max": int(np.max(rounds))},
        "listed_last": listed[-1],
        "roofline": {"bound": "hbm", "kernel": "k_sphere_steps", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "peak_source": which,
                     "bytes_per_launch": float(np.mean(b)), "ms_per_launch": total_ms / args.steps},
        "gpu_launches": int(launches),
        "iterations_to_residual": None,
        "picture": pic,
        "e2e": e2e,
    }
    line["clocks"] = clocks.summary()
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = sphere_cpu_baseline(scene, args.warmup, args.steps)
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


PILE_PUBLISHED_MS = {"until done mu=0.5": 3.04, "until done": 2.07, "grid averaged omega=1": 0.33}
PILE_WORKLOAD = ("sphere pile: the reference's large pile, 16^3 = 4,096 spheres r 3 cm dropped as a loose lattice "
                 "(java.util.Random(7) jitter), dt 1/60 s, 10 substeps of one pass; headline Gauss-Seidel run until "
                 "done with mu 0.5; also until done without friction and grid Jacobi (averaged); 240 frames, timed "
                 "2..239")


def run_sphere_pile(args):
    """The reference's own sphere benchmark scene (its sphere sweep's large pile) with its published solver
    settings: each solver's ms a step over the frames the reference times, the headline's line against its
    published laptop-GPU figure."""
    world_size, rank, local, pg = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from vxr import scenes
    from vxr import spheres as S
    from vxr.sphere_simulation import SphereSimulation

    def make(sc):
        sim = SphereSimulation(sc["spheres"], sc["substeps"], sc["iterations"], sc["grid"], sc["solve"], device=local,
                               blocks=args.sphere_blocks, cluster=args.sphere_cluster)
        sim.start(sc["x"], sc["y"], sc["z"], sc["u"], sc["v"], sc["w"], sc["r"], sc["im"], sc["params"])
        sim.friction(sc["friction"])
        return sim

    solvers, head = {}, None
    with Clocks(local) as clocks:
        for name in scenes.PILE_SOLVERS:
            sc = scenes.sphere_pile(seed=7 + rank, solver=name)
            n, frames = sc["spheres"], sc["frames"]
            sim = make(sc)
            stream = torch.cuda.ExternalStream(sim.stream())
            sim.step_and_wait(2)  # the reference's untimed first two frames
            launches0 = sim.launches()
            starts = [torch.cuda.Event(enable_timing=True) for _ in range(frames - 2)]
            ends = [torch.cuda.Event(enable_timing=True) for _ in range(frames - 2)]
            listed, rounds = [], []
            barrier(pg)
            torch.cuda.synchronize()
            for k in range(frames - 2):
                with torch.cuda.stream(stream):
                    starts[k].record(stream)
                sim.step_async(1)
                with torch.cuda.stream(stream):
                    ends[k].record(stream)
                rep = sim.sync()
                rounds.append(rep.rounds)
                listed.append(int(sim.counts()[S.LISTED]) if sc["solve"] != S.JACOBI else 0)
            torch.cuda.synchronize()
            barrier(pg)
            total_ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends)))
            slowest = all_max(pg, total_ms)
            entry = {"ms_per_step": slowest / (frames - 2), "published_laptop_ms": PILE_PUBLISHED_MS[name],
                     "speedup_vs_published": PILE_PUBLISHED_MS[name] / (slowest / (frames - 2)),
                     "rounds_per_step": float(np.mean(rounds)), "launches": int(sim.launches() - launches0)}
            if head is None:  # the headline: until done with friction
                head = {"scene": sc, "n": n, "frames": frames, "total_ms": slowest, "listed": listed,
                        "rounds": rounds, "launches": entry["launches"]}
            solvers[name] = entry
            sim.close()

    sc, n, timed = head["scene"], head["n"], head["frames"] - 2
    bodies_all = all_sum(pg, float(n))
    value = bodies_all * timed / (head["total_ms"] / 1e3)
    hbm, which = peaks()
    b = [sphere_step_bytes(n, sc["substeps"], sc["iterations"], min(l, 6 * n), r)
         for l, r in zip(head["listed"], head["rounds"])]
    achieved = sum(b) / (head["total_ms"] / 1e3) / 1e9
    e2e = None
    if not args.no_e2e:
        sim2 = make(sc)
        pinned = [torch.empty(n, dtype=torch.float32, pin_memory=True).numpy() for _ in range(9)]
        sim2.step_and_wait(2)
        sim2.state(pinned)
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(timed):
            sim2.params(sc["params"])
            sim2.step_and_wait(1)
            sim2.state(pinned)
        e2e_s = all_max(pg, time.perf_counter() - t0)
        sim2.close()
        e2e = {"value": bodies_all * timed / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 13 * 4,
               "d2h_bytes_per_step": 9 * 4 * n}
    published = n / (PILE_PUBLISHED_MS["until done mu=0.5"] / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": timed, "warmup": 2,
        "ms_per_step": head["total_ms"] / timed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / (published * world_size), "dtype": "f32", "data": "synthetic",
        "config": {"workload": PILE_WORKLOAD, "spheres": n, "substeps": sc["substeps"], "iterations": 1,
                   "timed_steps": f"2..{head['frames'] - 1}", "l2": "not flushed: the 4,096 spheres' state and list "
                   "(about 1 MB) live in L2 by design, as in the reference's own timing",
                   "parallelism": "replicas" if world_size > 1 else "single"},
        "vs_baseline_note": "the reference's published laptop-GPU (RTX 5070 Ti, Vulkan) time for this scene and solver, "
                            "3.04 ms a step; its host waits are included there, and the step is one launch here",
        "solvers": solvers,
        "roofline": {"bound": "hbm", "kernel": "k_sphere_steps", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "peak_source": which,
                     "bytes_per_launch": float(np.mean(b)), "ms_per_launch": head["total_ms"] / timed},
        "gpu_launches": head["launches"],
        "e2e": e2e,
    }
    line["clocks"] = clocks.summary()
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = pile_cpu_baseline(sc, warm=2, steps=timed)
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def pile_cpu_baseline(sc, warm=2, steps=238):
    """The serial oracle on the pile with the headline solver: frames warm..warm+steps-1, timed on the host."""
    from oracle.sphere import OracleSphereWorld
    from vxr import spheres as S
    w = OracleSphereWorld(sc["spheres"], sc["substeps"], sc["iterations"], sc["solve"], sc["grid"])
    for k in ("x", "y", "z", "u", "v", "w", "r", "im"):
        w.set_field(k, sc[k])
    w.set_shown(S.shown_at_start(sc["x"], sc["y"], sc["z"], sc["r"]))
    w.set_params(sc["params"], sc["friction"])
    w.step(warm)
    t0 = time.perf_counter()
    w.step(steps)
    dt = time.perf_counter() - t0
    w.close()
    return {"value": sc["spheres"] * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"the whole pile, frames {warm}..{warm + steps - 1}, {dt:.1f} s, serial C++ oracle"}


BATCH_WORKLOAD = ("batched scenes: 512 independent scenes, bodies log-U[64,4096] each (70% spheres / 30% boxes, the "
                  "large mixed scene's size distributions), per-scene gravity tilt U(+-5 deg) and mu U[0.3,0.8], "
                  "dt 1/60 s, 4 substeps, 10 sweeps; one world, steps replayed from a captured CUDA graph")


def batch_subset(b, scenes_idx):
    """The scenes `scenes_idx` of a batch, as a batch of their own."""
    from vxr import scenes
    parts = [b["parts"][k] for k in scenes_idx]
    out = {name: np.concatenate([p[name] for p in parts]) for name in scenes.FIELDS}
    out.update({"counts": np.asarray([b["counts"][k] for k in scenes_idx], np.int32),
                "grids": [b["grids"][k] for k in scenes_idx], "walls": [b["walls"][k] for k in scenes_idx],
                "params": b["params"][list(scenes_idx)], "parts": parts, "substeps": b["substeps"],
                "sweeps": b["sweeps"], "scenes": len(parts)})
    out["bodies"] = int(out["counts"].sum())
    return out


def batch_cpu_baseline(b, warm=2, steps=24, scenes_wanted=16):
    """The OpenMP oracle on a bounded sample of the batch: its first scenes, each a world of its own."""
    from oracle.box import OracleBoxWorld, lib as orc_lib
    from vxr import scenes
    picked = list(range(min(scenes_wanted, len(b["parts"]))))
    worlds = []
    for k in picked:
        part = b["parts"][k]
        w = OracleBoxWorld(part["bodies"], part["substeps"], part["sweeps"], False, part["grid"], threads=True)
        for name in scenes.FIELDS:
            w.set_field(name, part[name])
        w.set_params(b["params"][k])
        w.step(warm)
        worlds.append(w)
    t0 = time.perf_counter()
    for w in worlds:
        w.step(steps)
    dt = time.perf_counter() - t0
    bodies = sum(b["parts"][k]["bodies"] for k in picked)
    for w in worlds:
        w.close()
    return {"value": bodies * steps / dt, "unit": UNIT, "cores": int(orc_lib(True).orc_threads()), "kind": "port",
            "sample": f"the first {len(picked)} scenes ({bodies} bodies), steps {warm}..{warm + steps - 1}, {dt:.1f} s, "
                      "OpenMP C++ oracle, scene after scene"}


def run_batched(args):
    """Batched scenes: one world of every scene (this rank's share), stepped by CUDA graph replays."""
    world_size, rank, local, pg = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from vxr import autotune, scenes
    from vxr.box_simulation import BatchSimulation
    full = scenes.batched(seed=1)
    mine = shard_scenes(full["scenes"], world_size, rank)  # scenes shared out across the ranks
    b = batch_subset(full, mine) if world_size > 1 else full
    tune = autotune.tune_batch(b, local)
    grids = autotune.scaled_grids(b, tune["cell_scale"])

    def make():
        sim = BatchSimulation(b["counts"], grids, b["substeps"], b["sweeps"], device=local,
                              schedule=tune["schedule"], solve_blocks_per_sm=tune["solve_blocks_per_sm"])
        sim.load_state([b[k] for k in scenes.FIELDS], None)
        sim.scene_params(b["params"])
        sim.islands(tune.get("islands", True))
        return sim

    sim = make()
    stream = torch.cuda.ExternalStream(sim.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    sim.step_and_wait(args.warmup)
    sim.step_graph(1)  # capture the graph outside the timed region
    sim.sync()
    pairs = max(1, args.steps // 2)
    launches0 = sim.launches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(pairs)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(pairs)]
    reports = Reports()
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clocks:
        for k in range(pairs):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            sim.step_graph(1)
            with torch.cuda.stream(stream):
                ends[k].record(stream)
            if k % 10 == 9:
                reports.add(sim.sync())
        reports.finish(sim, 10, pairs)
    torch.cuda.synchronize()
    barrier(pg)
    launches = sim.launches() - launches0
    total_ms = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    steps = 2 * pairs
    slowest_ms = all_max(pg, total_ms)
    bodies_all = all_sum(pg, float(b["bodies"]))
    value = bodies_all * steps / (slowest_ms / 1e3)
    # the solve kernel's share, from a short profiled run of plain steps after the timed region
    sim.profile(True)
    sim.step_and_wait(10)
    phases = sim.profile(False)
    activity = sim.activity()
    solve_ms = phases[3] / 10
    hbm, which = peaks()
    b_solve = algorithmic_solve_bytes(b["bodies"], b["substeps"], b["sweeps"], activity["touching"],
                                      activity["points"], activity["bodies_active"], activity["wall_records"])
    achieved = b_solve / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    sim.close()
    e2e = None
    if not args.no_e2e:
        sim2 = make()
        # the step's result read into pinned host arrays, reused every step
        pinned = [torch.empty(b["bodies"], dtype=torch.float32, pin_memory=True).numpy() for _ in range(13)]
        for _ in range(args.warmup):
            sim2.step_and_wait(1)
            sim2.state(pinned)
        barrier(pg)
        e2e_steps = args.steps  # the same number of steps as the timed region, from the same start
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            sim2.scene_params(b["params"])
            sim2.step_and_wait(1)
            sim2.state(pinned)
        e2e_s = all_max(pg, time.perf_counter() - t0)
        sim2.close()
        e2e = {"value": bodies_all * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 18 * 4 * b["scenes"],
               "d2h_bytes_per_step": 13 * 4 * b["bodies"], "steps": e2e_steps}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": steps,
        "warmup": args.warmup, "ms_per_step": slowest_ms / steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "scenes": b["scenes"], "bodies": b["bodies"],
                   "timed_steps": f"{args.warmup + 2}..{args.warmup + 1 + steps}, as {pairs} replays of a two-step graph",
                   "l2": "flushed (256 MiB write) before every replay",
                   "autotuned": {k: tune.get(k) for k in ("cell_scale", "solve_blocks_per_sm", "schedule", "islands",
                                                          "cached")},
                   "parallelism": f"scenes shared out over {world_size} ranks" if world_size > 1 else "single"},
        "phase_ms_per_step": {"broad": phases[0] / 10, "narrow": phases[1] / 10, "colour": phases[2] / 10,
                              "solve": solve_ms},
        "last_step": {**reports.last_step(), **activity},
        "roofline": {"bound": "hbm", "kernel": "k_solve", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "peak_source": which, "bytes_per_launch": b_solve,
                     "ms_per_launch": solve_ms},
        "gpu_launches": int(launches),
        "e2e": e2e,
    }
    line["clocks"] = clocks.summary()
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = batch_cpu_baseline(b)
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


TOWERS_WORKLOAD = ("box stacking: 64 towers of 64 boxes (4,096) on an 8x8 grid at 3 m, half-extents U[0.25,0.75] m, "
                   "yaw U(+-15 deg), offset U(+-0.02) m; mu 0.6, no restitution; dt 1/60 s, 8 substeps, 16 sweeps")


def judged_run(sc, steps, every, device):
    """The configuration's run from its start, judged by the GPU's diagnostics every `every` steps: the deepest
    contact and wall penetration seen, the energy (kinetic with spin, plus potential) at the start, the end and its
    greatest rise, and bodies gone non-finite."""
    from vxr import learned as Lm
    j = Lm.settled_world(sc, 0, sc["sweeps"], device=device)
    d0 = j.gpu_diagnostics()
    e0 = d0["kinetic"] + d0["potential"]
    worst_pen, worst_wall, energy, broken = 0.0, 0.0, [], False
    t0 = time.perf_counter()
    for _ in range(steps // every):
        j.step_and_wait(every)
        d = j.gpu_diagnostics()
        worst_pen = max(worst_pen, d["max_penetration"])
        worst_wall = max(worst_wall, d["max_wall_penetration"])
        energy.append(d["kinetic"] + d["potential"])
        broken = broken or bool(d["broken"])
    top = float(np.max(j.field("y")))
    j.close()
    return {"steps": steps, "every": every, "max_penetration_start_m": d0["max_penetration"],
            "max_penetration_m": worst_pen, "max_wall_penetration_m": worst_wall,
            "energy_start_J": e0, "energy_end_J": energy[-1], "energy_drift": (energy[-1] - e0) / abs(e0),
            "energy_max_rise": (max(energy) - e0) / abs(e0), "highest_top_m": top, "broken": broken,
            "seconds": time.perf_counter() - t0}


def run_towers(args):
    """Box stacking: K timed steps; then the configuration's 1,000 steps judged by penetration and energy drift
    (the GPU's diagnostics every 10 steps)."""
    world_size, rank, local, pg = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from vxr import learned as Lm
    from vxr import scenes
    sc = scenes.towers(seed=1 + rank)
    n = sc["bodies"]
    w = Lm.settled_world(sc, 0, sc["sweeps"], device=local)
    stream = torch.cuda.ExternalStream(w.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    w.step_and_wait(args.warmup)
    launches0 = w.launches()
    w.profile(True)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    reports = Reports()
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            w.step_async(1)
            with torch.cuda.stream(stream):
                ends[k].record(stream)
            if k % 20 == 19:
                reports.add(w.sync())
        reports.finish(w, 20, args.steps)
    torch.cuda.synchronize()
    barrier(pg)
    phases = w.profile(False)
    activity = w.activity()
    launches = w.launches() - launches0
    total_ms = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    slowest_ms = all_max(pg, total_ms)
    value = all_sum(pg, float(n)) * args.steps / (slowest_ms / 1e3)
    solve_ms = phases[3] / args.steps
    hbm, which = peaks()
    b_solve = algorithmic_solve_bytes(n, sc["substeps"], sc["sweeps"], activity["touching"], activity["points"],
                                      activity["bodies_active"], activity["wall_records"])
    achieved = b_solve / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    pic = picture_timing(w, 1, n, sc["walls"], local, squash=0.0, cpu=rank == 0 and not args.no_cpu)
    w.close()
    judged = judged_run(sc, 1000, 10, local)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": slowest_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": TOWERS_WORKLOAD, "bodies": n, "substeps": sc["substeps"], "sweeps": sc["sweeps"],
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": "replicas" if world_size > 1 else "single"},
        "judged_1000_steps": judged,
        "picture": pic,
        "phase_ms_per_step": {"broad": phases[0] / args.steps, "narrow": phases[1] / args.steps,
                              "colour": phases[2] / args.steps, "solve": solve_ms},
        "last_step": {**reports.last_step(), **activity},
        "roofline": {"bound": "hbm", "kernel": "k_solve", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "peak_source": which, "bytes_per_launch": b_solve,
                     "ms_per_launch": solve_ms},
        "gpu_launches": int(launches),
    }
    line["clocks"] = clocks.summary()
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_reference(args):
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return 0
    if args.workload == "batched-scenes":
        from vxr import scenes
        base = batch_cpu_baseline(scenes.batched(seed=1), warm=min(args.warmup, 3), steps=min(args.steps, 24))
        line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
                "steps": min(args.steps, 24), "warmup": min(args.warmup, 3), "ms_per_step": None,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": BATCH_WORKLOAD}, "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    if args.workload == "sphere-pile":
        from vxr import scenes
        sc = scenes.sphere_pile()
        steps = max(1, min(args.steps, sc["frames"] - 2))  # the frames the reference times, at most
        base = pile_cpu_baseline(sc, warm=2, steps=steps)
        line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
                "steps": steps, "warmup": 2, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": PILE_WORKLOAD, "spheres": sc["spheres"]}, "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    if args.workload == "sphere-lattice":
        from vxr import scenes
        scene = scenes.sphere_lattice()
        base = sphere_cpu_baseline(scene, min(args.warmup, 3), args.steps)
        line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": min(args.warmup, 3), "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": SPHERE_WORKLOAD, "spheres": scene["spheres"]}, "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    steps = min(args.steps, 24)
    warm = min(args.warmup, 3)
    base = cpu_baseline(steps_timed=steps, warm=warm)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "large mixed scene (262,144 bodies, 80% spheres / 20% boxes), bounded "
                                   "1/16-volume sample per step", "bodies": BODIES, "substeps": 4, "sweeps": 10,
                       "dt": 1 / 120},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (Java on the SupirVast IR) cannot run here; its CPU path is restated as the "
                    "C++ oracle, timed with every host thread"}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vxr", choices=["vxr", "reference"])
    ap.add_argument("--bodies", type=int, default=BODIES)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-iterations", action="store_true")
    ap.add_argument("--no-judge", action="store_true", help="skip the judged run (penetration, energy)")
    ap.add_argument("--schedule", type=int, default=0, help="solve schedule: 0 barrier phases, 1 per-body dependencies")
    ap.add_argument("--sphere-blocks", type=int, default=0, help="sphere workloads: blocks (0: the library's choice)")
    ap.add_argument("--sphere-cluster", type=int, default=0, help="sphere workloads: cluster size (0: the library's)")
    ap.add_argument("--save-state", default="", help="large scene: save the state after the warm-up steps and exit")
    ap.add_argument("--load-state", default="", help="large scene: start from a state saved by --save-state")
    ap.add_argument("--solve-blocks-per-sm", type=int, default=0, help="solve blocks an SM (0: the library's choice)")
    ap.add_argument("--max-pairs", type=int, default=0, help="pair capacity of the world (0: 32 a body)")
    ap.add_argument("--cell", type=float, default=0.0,
                    help="large scene: grid cell in metres (0: the reference's rule, about 2.07 m); a narrower cell "
                         "walks as many cells each way as the rule's width needs (1.6 m: 2, the 125 cells)")
    ap.add_argument("--no-landed", action="store_true", help="large scene: skip the landed-pile window")
    ap.add_argument("--no-islands", action="store_true",
                    help="every body through the grid-wide phases (small components not solved by island blocks)")
    ap.add_argument("--list-kernel", default="thread", choices=["thread", "tiled"],
                    help="large scene: the broad phase's list, a thread a body (default) or tiles of cells staged in "
                         "shared memory; both list the same pairs")
    ap.add_argument("--workload", default="large-mixed",
                    choices=["large-mixed", "sphere-lattice", "batched-scenes", "towers", "sphere-pile"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "sphere-lattice":
        return run_spheres(args)
    if args.workload == "batched-scenes":
        return run_batched(args)
    if args.workload == "towers":
        return run_towers(args)
    if args.workload == "sphere-pile":
        return run_sphere_pile(args)

    world_size, rank, local, pg = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from vxr import scenes

    if args.bodies == BODIES:
        scene = scenes.large_mixed(args.bodies, seed=1 + rank)
    else:  # a smaller case of the same scene: the same body density over a smaller footprint
        scene = scenes.sub_volume(BODIES, args.bodies / BODIES, seed=1 + rank)
    if args.cell > 0:
        with_cell(scene, args.cell)
    w = make_world(scene, local, args.max_pairs, args.schedule, args.solve_blocks_per_sm, not args.no_islands)
    w.list_kernel(args.list_kernel == "tiled")
    if args.load_state:  # a state saved by --save-state: the 13 moving fields; shapes, masses and params the scene's
        z = np.load(args.load_state)
        moving = [z[f"arr_{i}"] for i in range(13)]
        w.load_state(moving + [scene["im"], scene["hx"], scene["hy"], scene["hz"], scene["shape"]], scene["params"])
    stream = torch.cuda.ExternalStream(w.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    # warm-up: steps 0..W-1
    w.step_async(args.warmup)
    w.sync()
    if args.save_state:  # the state after the warm-up steps, for a later run (or a profile of one late step)
        np.savez(args.save_state, *w.state())
        if rank == 0:
            print(json.dumps({"saved": args.save_state, "after_steps": args.warmup, "touching": w.last().touching}))
        w.close()
        if pg is not None:
            pg.destroy_process_group()
        return 0
    launches0 = w.launches()
    w.profile(True)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampled = []
    reports = Reports()
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            w.step_async(1)
            with torch.cuda.stream(stream):
                ends[k].record(stream)
            if k % 20 == 19:
                reports.add(w.sync())
                # the solve's algorithmic bytes, sampled every 20th step at the sync the loop makes anyway
                a = w.activity()
                sampled.append(algorithmic_solve_bytes(scene["bodies"], scene["substeps"], scene["sweeps"],
                                                       a["touching"], a["points"], a["bodies_active"],
                                                       a["wall_records"]))
        reports.finish(w, 20, args.steps)
    torch.cuda.synchronize()
    barrier(pg)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    phases = w.profile(False)
    launches = w.launches() - launches0
    activity = w.activity()
    total_ms = float(sum(step_ms))
    slowest_ms = all_max(pg, total_ms)
    bodies_all = all_sum(pg, float(scene["bodies"]))
    value = bodies_all * args.steps / (slowest_ms / 1e3)
    # the drop's phases: body-steps/s over windows of 100 timed steps (this rank's own events)
    windows = []
    for lo in range(0, args.steps, 100):
        ms = float(sum(step_ms[lo:lo + 100]))
        hi = min(lo + 100, args.steps)
        windows.append({"steps": f"{args.warmup + lo}..{args.warmup + hi - 1}", "ms_per_step": ms / (hi - lo),
                        "value": scene["bodies"] * (hi - lo) / (ms / 1e3)})

    # roofline of the solve kernel: algorithmic bytes per launch averaged over the timed steps (sampled every 20th),
    # over its mean launch time from the per-phase events
    hbm, which = peaks()
    solve_ms = phases[3] / args.steps
    if not sampled:
        sampled.append(algorithmic_solve_bytes(scene["bodies"], scene["substeps"], scene["sweeps"],
                                               activity["touching"], activity["points"], activity["bodies_active"],
                                               activity["wall_records"]))
    b_solve = float(np.mean(sampled))
    # the measured traffic belongs to the timed window only where that window is the default run's early drop
    default_window = args.warmup <= 10 and not args.load_state and not args.no_islands and args.cell <= 0
    achieved = b_solve / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    pic = picture_timing(w, 1, scene["bodies"], scene["walls"], local, squash=0.0,
                         cpu=rank == 0 and not args.no_cpu)

    # The timed steps' quality: a second world along the same trajectory (the step is deterministic and measuring
    # changes no result), stepped untimed to the timed window's start, then the same steps measured.
    wq = make_world(scene, local, args.max_pairs, args.schedule, args.solve_blocks_per_sm, not args.no_islands)
    wq.step_and_wait(args.warmup)
    quality = window_quality(wq, scene, args.steps)
    quality["same_trajectory_as_timed"] = all(np.array_equal(a.view(np.int32), b.view(np.int32))
                                              for a, b in zip(wq.state(), w.state()))
    wq.close()

    # The landed pile: the scene stepped untimed to LANDED_STEP (bodies from the top of the volume land about then),
    # then as many steps as the timed window, timed the same way, and their quality measured on the steps after.
    landed, wl = None, None
    if not args.no_landed:
        wl = make_world(scene, local, args.max_pairs, args.schedule, args.solve_blocks_per_sm, not args.no_islands)
        for _ in range(LANDED_STEP // 20):
            wl.step_async(20)
            wl.sync()
        with Clocks(local) as clocks_l:  # its clocks join the timed window's record
            ms_l = timed_steps(wl, torch.cuda.ExternalStream(wl.stream), flush, args.steps)
        clocks.samples += clocks_l.samples
        slow_l = all_max(pg, float(sum(ms_l)))
        landed = {"steps": f"{LANDED_STEP}..{LANDED_STEP + args.steps - 1}", "ms_per_step": slow_l / args.steps,
                  "value": bodies_all * args.steps / (slow_l / 1e3), "touching": wl.last().touching,
                  "rounds": wl.last().rounds, "paths": wl.paths(),
                  "quality": window_quality(wl, scene, min(args.steps, 10))}

    # Iterations to residual: the pile as the timed steps left it, a substep's solve sweeps run until a sweep's
    # residual (the largest positional correction it makes at any contact point) is 1e-4 m or less, at most 64; with
    # the impulses carried from the step before (the reference's warm start), from zero, and from the learned warm
    # start's network, each start on the same steps. The network is trained first, on the GPU, on 2M contact points of
    # two other worlds of the same distribution, its targets the impulses the plain solver reached run to a residual
    # of 1e-6 m (at most 64 sweeps); the plain solver then judges it, and it is kept only if it gains.
    iters = {"tolerance_m": 1e-4, "cap": ITERATION_CAP, "definition": "solve sweeps a substep runs until its residual "
             "max_points h k (|dlambda_n| + |dlambda_t|) <= 1e-4 m"}
    if not args.no_iterations:
        from vxr import learned as Lm
        t0 = time.perf_counter()
        def train_scene(seed):
            if args.bodies == BODIES:
                return scenes.large_mixed(args.bodies, seed=seed + rank)
            return scenes.sub_volume(BODIES, args.bodies / BODIES, seed=seed + rank)
        # 2M rows from two other worlds of the same distribution, at the two phases the judgement looks at: the early
        # drop (settled as far as the timed window) and the landed pile
        plan = [(train_scene(101), args.warmup + args.steps)]
        if not args.no_landed:
            plan.append((train_scene(102), LANDED_STEP))
        feats, targets, _ = Lm.gather_many(plan, rows_wanted=2_000_000, sweeps_cap=ITERATION_CAP, tolerance=1e-6,
                                           device=local)
        gather_s = time.perf_counter() - t0
        # one row in ten held out: the network's accuracy against the carried impulses and against zero. It is trained
        # on the points that carried nothing, the ones its start is kept for (mode 3)
        held = np.arange(len(feats)) % 10 == 9
        use = ~held & Lm.new_contacts(feats)
        net = Lm.Mlp(device=local, seed=7)
        t1 = time.perf_counter()
        losses = net.train(feats[use], targets[use], epochs=20, batch=4096, lr=1e-3, seed=8)
        train_s = time.perf_counter() - t1
        accuracy = Lm.prediction_errors(net, feats[held], targets[held])
        # judged on twins of the timed world (and of the landed one): every start takes the same three steps, from
        # the carried impulses, from zero, from the network, and from the answers a perfect predictor would give (the
        # impulses the step, or its first substep alone, reaches solved to 1e-6 m)
        t2 = time.perf_counter()
        verdict = Lm.judge(scene, w.state(), net, samples=3, tolerance=1e-4, cap=ITERATION_CAP, ceiling=True,
                           device=local)
        if wl is not None:
            landed["iterations_to_residual"] = Lm.judge(scene, wl.state(), net, samples=3, tolerance=1e-4,
                                                        cap=ITERATION_CAP, ceiling=True, device=local)
        judge_s = time.perf_counter() - t2
        net.close()
        w.measure(residual=False, cold_start=False, sweeps=scene["sweeps"], tolerance=0.0)
        iters.update(verdict)
        iters["training"] = {"rows": int(len(feats)), "trained_on": int(use.sum()),
                             "trained_on_what": "the new contacts (points that carried nothing) of the rows not held out",
                             "epochs": 20, "batch": 4096,
                             "lr": 1e-3, "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
                             "gather_s": gather_s, "train_s": train_s, "judge_s": judge_s,
                             "data": "two other worlds of the same distribution (seeds 101 and 102), one settled as far "
                                     "as the timed window, one to the landed pile; targets from the plain solver run "
                                     "to 1e-6 m (at most 64 sweeps)",
                             "held_out_rms_scaled": accuracy}

    if wl is not None:
        wl.close()
    judged = None
    if not args.no_judge:
        judged = judged_run(scene, 500, 10, local)

    e2e = None
    if not args.no_e2e:
        w2 = make_world(scene, local, args.max_pairs, args.schedule, args.solve_blocks_per_sm, not args.no_islands)
        # each step's result read into pinned host arrays, two sets used in turn: step k's state is split on the
        # device and copied out on a stream of its own while step k + 1 runs, and the loop waits for step k's copy
        # before it goes past step k + 1. Every step's 13 fields reach host memory inside the timed region.
        pinned = [[torch.empty(scene["bodies"], dtype=torch.float32, pin_memory=True).numpy() for _ in range(13)]
                  for _ in range(2)]
        for _ in range(args.warmup):
            w2.step_and_wait(1)
            w2.state(pinned[0])
        barrier(pg)
        t0 = time.perf_counter()
        for k in range(args.steps):
            w2.params(scene["params"])
            w2.step_async(1)
            w2.state_async(pinned[k % 2], k % 2)
            if k > 0:
                w2.state_wait((k - 1) % 2)
            if k % 20 == 19:
                w2.sync()  # the steps' reports (an error status raises)
        w2.state_wait((args.steps - 1) % 2)
        w2.sync()
        e2e_s = time.perf_counter() - t0
        w2.close()
        e2e_s = all_max(pg, e2e_s)
        e2e = {"value": bodies_all * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 18 * 4,
               "d2h_bytes_per_step": 13 * 4 * scene["bodies"],
               "read_back": "every step's state into pinned host arrays, copied on a second stream while the next "
                            "step runs (vxr_box_state_async / vxr_box_state_wait)"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": slowest_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"large mixed scene: {scene['bodies']} bodies, 80% spheres r log-U[0.2,0.8] m, "
                               "20% boxes half U[0.2,0.6] m, 128x64x128 m drop, v N(0,1), rho U[500,2000]",
                   "bodies": scene["bodies"], "dt": scene["dt"], "substeps": scene["substeps"],
                   "sweeps": scene["sweeps"], "mu": scene["mu"], "mu_rolling": scene["mu_rolling"],
                   "grid": [scene["grid"].nx, scene["grid"].ny, scene["grid"].nz, scene["grid"].cell],
                   "reach_cells": scene.get("reach_cells", 1),
                   "timed_steps": f"{args.warmup}..{args.warmup + args.steps - 1} of the drop",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "schedule": args.schedule, "solve_blocks_per_sm": args.solve_blocks_per_sm,
                   "list_kernel": args.list_kernel,
                   "parallelism": "replicas" if world_size > 1 else "single"},
        "phase_ms_per_step": {"broad": phases[0] / args.steps, "narrow": phases[1] / args.steps,
                              "colour": phases[2] / args.steps, "solve": phases[3] / args.steps},
        "windows": windows,
        "last_step": {**reports.last_step(), **activity},
        "roofline": {"bound": "hbm", "kernel": "the solve (k_islands, then k_solve)", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "traffic": EARLY_SOLVE_TRAFFIC["dram_bytes"] if args.bodies == BODIES and default_window else None,
                     "peak_source": which, "bytes_per_launch": b_solve, "ms_per_launch": solve_ms,
                     "bytes_per_launch_sampled": "every 20th timed step",
                     "traffic_launch": EARLY_SOLVE_TRAFFIC if args.bodies == BODIES and default_window else None,
                     "traffic_late_launch": LATE_SOLVE_TRAFFIC if args.bodies == BODIES else None},
        "gpu_launches": int(launches),
        "iterations_to_residual": iters,
        "quality": quality,
        "landed_window": landed,
        "judged_500_steps": judged,
        "picture": pic,
        "e2e": e2e,
    }
    line["clocks"] = clocks.summary()
    if rank == 0 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline()
        except Exception as e:  # the baseline is reported, not required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(e)}
    w.close()
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
