"""The multi-rank host logic of bench.py on CPU: two ranks over gloo (127.0.0.1), as torchrun starts them. The
whole-job rate sums the ranks' bodies over the slowest rank's time; the batched scenes are shared out with no scene
on two ranks and none left over; and each rank's share of a real batch is a batch of its own with the right
bodies."""
import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "vexelray-sim-rigid_b200"))
    import bench
    from vxr import scenes
    res = {}
    res["max"] = bench.all_max(dist, 1.0 + rank)
    res["sum"] = bench.all_sum(dist, 1.0 + rank)
    # rank 1 is the slow one: 150 ms against 100
    res["rate"] = bench.whole_job_rate(dist, 1000 + 24 * rank, 10, 100.0 + 50.0 * rank)
    res["mine"] = bench.shard_scenes(37, world, rank)
    full = scenes.batched(scenes=6, seed=3, smallest=64, largest=200)
    part = bench.batch_subset(full, bench.shard_scenes(full["scenes"], world, rank))
    res["part_bodies"] = part["bodies"]
    res["part_counts"] = part["counts"].tolist()
    res["part_x0"] = float(part["x"][0])
    res["full_counts"] = full["counts"].tolist()
    res["full_first_x"] = [float(full["parts"][k]["x"][0]) for k in range(full["scenes"])]
    bench.barrier(dist)
    dist.destroy_process_group()
    out[rank] = res


def test_two_ranks_over_gloo():
    world = 2
    with mp.get_context("spawn").Manager() as m:  # spawned, never forked from a threaded process
        out = m.dict()
        mp.spawn(rank_main, args=(world, free_port(), out), nprocs=world, join=True)
        res = [out[r] for r in range(world)]
    for r in res:
        assert r["max"] == 2.0 and r["sum"] == 3.0
        assert np.isclose(r["rate"], (1000 + 1024) * 10 / 0.150)
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(37))
    assert not set(res[0]["mine"]) & set(res[1]["mine"])
    counts = res[0]["full_counts"]
    for rank, r in enumerate(res):
        want = [counts[k] for k in range(len(counts)) if k % world == rank]
        assert r["part_counts"] == want
        assert r["part_bodies"] == sum(want)
        assert r["part_x0"] == r["full_first_x"][rank]
