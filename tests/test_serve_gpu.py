"""The serving loop (steel_serve_*): requests for different instances of one batch, admitted a few
at a time, give every instance exactly the result it has when run alone for the same frames."""
import numpy as np
import pytest

from steel_webgpu_b200 import pack
from steel_webgpu_b200.sim import Batch, Server
from tests import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _state(batch, scene):
    return [_bits(x) for x in batch.raw_state(scene)]


def test_served_instances_match_running_alone(steel):
    pks = [pack(s) for s in scenes.small_batch(seed=21, n=6)]
    b = Batch(pks)
    srv = Server(b, max_active=3)
    plan = {0: [5], 1: [2, 3], 3: [7], 4: [1, 1, 1]}  # instance -> frames of its requests, in order
    ids = {}
    for inst, reqs in plan.items():
        for frames in reqs:
            ids[srv.submit(inst, frames)] = inst
    done, ticks = [], 0
    while len(done) < len(ids):
        assert srv.tick() <= 3
        done += srv.poll()
        ticks += 1
        assert ticks < 100
    assert sorted(d[0] for d in done) == sorted(ids)
    assert all(ids[rid] == inst and lat >= 0.0 for rid, inst, lat in done)
    total = {i: sum(r) for i, r in plan.items()}
    for i, pk in enumerate(pks):
        alone = Batch([pk])
        if total.get(i, 0):
            alone.step(total[i])
        for got, ref in zip(_state(b, i), _state(alone, 0)):
            assert np.array_equal(got, ref), f"instance {i} differs from running alone"
        alone.close()
    # After the loop ends every scene steps again.
    srv.close()
    b.step(1)
    alone = Batch([pks[2]])
    alone.step(1)
    for got, ref in zip(_state(b, 2), _state(alone, 0)):
        assert np.array_equal(got, ref)
    alone.close()
    b.close()


def test_budget_admission_and_compacted_launches(steel):
    """Admission by bytes: with a budget of the two largest instances' state, at most that much is
    admitted per tick (the head of the queue always when nothing is); the per-scene kernels launch
    only the admitted instances, and every instance still matches running alone."""
    pks = [pack(s) for s in scenes.small_batch(seed=23, n=6)]
    b = Batch(pks)
    sizes = [b.scene_bytes(i) for i in range(len(pks))]
    budget = sorted(sizes)[-1] + sorted(sizes)[-2]
    srv = Server(b, budget_bytes=budget)
    frames = {i: 3 + i for i in range(len(pks))}
    for i, f in frames.items():
        srv.submit(i, f)
    done, ticks = [], 0
    while len(done) < len(pks):
        n = srv.tick()
        assert n >= 1
        done += srv.poll()
        ticks += 1
        assert ticks < 200
    srv.close()
    for i, pk in enumerate(pks):
        alone = Batch([pk])
        alone.step(frames[i])
        for got, ref in zip(_state(b, i), _state(alone, 0)):
            assert np.array_equal(got, ref), f"instance {i} differs from running alone"
        alone.close()
    b.close()
