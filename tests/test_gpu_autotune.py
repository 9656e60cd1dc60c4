"""The batched scenes' autotuner (vxr/autotune.py): every candidate it times steps a batch to the same bits, so its
choice changes speed only; its cache separates batch shapes and a cached choice is reused without a search."""
import os

import numpy as np
import pytest

from vxr import autotune, scenes


def small_batch():
    return scenes.batched(scenes=12, seed=4, smallest=64, largest=600)


def test_the_cache_key_separates_batch_shapes():
    a = small_batch()
    b = scenes.batched(scenes=12, seed=5, smallest=64, largest=600)
    c = dict(a, substeps=a["substeps"] + 1)
    keys = {autotune._key(x, "B200") for x in (a, b, c)}
    assert len(keys) == 3
    assert autotune._key(a, "B200") != autotune._key(a, "H100")
    assert len(autotune.candidates()) == (len(autotune.CELL_SCALES) * len(autotune.BLOCKS_PER_SM) *
                                          len(autotune.SCHEDULES) * len(autotune.ISLANDS))


@pytest.mark.gpu
def test_every_candidate_steps_the_batch_to_the_same_bits():
    b = small_batch()
    first = autotune.make_batch(b, (1.0, 0, 0, True))
    first.step_and_wait(30)  # bodies landing: pairs, walls and components of every size
    state = first.state()
    first.close()
    results = []
    for cand in autotune.candidates():
        sim = autotune.make_batch(b, cand, state)
        sim.step_and_wait(8)
        results.append((cand, sim.state()))
        sim.close()
    want = results[0][1]
    for cand, got in results[1:]:
        for x, y in zip(got, want):
            assert np.array_equal(x.view(np.int32), y.view(np.int32)), cand


@pytest.mark.gpu
def test_a_cached_choice_is_reused(tmp_path, monkeypatch):
    monkeypatch.setenv("VXR_TUNE_CACHE", os.path.join(str(tmp_path), "tune.json"))
    b = small_batch()
    one = autotune.tune_batch(b, settle_steps=10, warm_steps=1, timed_steps=2)
    assert one["cached"] is False and len(one["trials"]) == len(autotune.candidates())
    two = autotune.tune_batch(b, settle_steps=10, warm_steps=1, timed_steps=2)
    assert two["cached"] is True
    for k in ("cell_scale", "solve_blocks_per_sm", "schedule", "islands"):
        assert two[k] == one[k]
    other = autotune.tune_batch(scenes.batched(scenes=10, seed=6, smallest=64, largest=400), settle_steps=10,
                                warm_steps=1, timed_steps=2)
    assert other["cached"] is False
