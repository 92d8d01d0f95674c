"""Every scene folder the reference ships (assets/scenes/*), packed as the reference packs it,
stepped by the CUDA path through the C ABI and by the oracle side by side.

Poses, velocities, joint coordinates and joint velocities are compared bit for bit every 60 frames
(240 frames per scene, 1020 for the scenes that step cheaply on the oracle), and the stats words
(contacts, colors, max pairs, max units) with them. When a checkpoint differs, the scene is
replayed to the last agreeing checkpoint and then stepped one kernel at a time on both sides to
name the first stage whose output differs.

The packed scenes come from tests/golden/make_reference_scenes.py (run by the build where the
reference is checked out); the GPU box gets them with the working tree.
"""
import multiprocessing as mp
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import pytest

from steel_webgpu_b200.sim import Batch
from tests import refscenes

pytestmark = pytest.mark.gpu
NAMES = refscenes.names()


@pytest.fixture(scope="module")
def oracle_runs(oracle_lib):
    """Oracle checkpoints of every scene, computed in spawned processes (the slowest first)."""
    import os
    slow = ["lava_fall", "cereal", "brick_pour", "bolt_sweep", "dominoes", "trebuchet", "cup_unpacking"]
    order = sorted(NAMES, key=lambda n: (n not in slow, slow.index(n) if n in slow else 0, n))
    ex = ProcessPoolExecutor(max_workers=max(2, min(24, (os.cpu_count() or 4) - 1)), mp_context=mp.get_context("spawn"))
    futs = {n: ex.submit(refscenes.oracle_checkpoints, n) for n in order}
    yield futs
    ex.shutdown(wait=True, cancel_futures=True)


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _first_difference(pk, good_frames, oracle_lib):
    """Replays both sides to `good_frames`, then steps substep by substep, comparing after each
    kernel group; returns a description of the first stage whose output differs."""
    C = pk.C
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    if good_frames:
        o.step(good_frames)
        g.step(good_frames)
    for sub in range(refscenes.EVERY * pk.params["substeps"]):
        o.stage(0)
        g.debug_stage(0)
        o.stage(1)
        g.debug_stage(1)
        osch = o.read("sched", np.uint32)
        nu = osch[C["S_META"]]
        tot = osch[C["S_USTART"] + nu]
        if g.read_words("sched", g.layout("S_META"), 2, dtype=np.uint32).tolist() != [nu, osch[C["S_META"] + 1]]:
            return f"substep {sub} after frame {good_frames}: unit/color counts (prepare)"
        gcol = g.read_words("sched", g.layout("S_PCOL"), tot, dtype=np.uint32)
        if not np.array_equal(gcol, osch[C["S_PCOL"]:C["S_PCOL"] + tot]):
            return f"substep {sub} after frame {good_frames}: colors (prepare)"
        if not np.array_equal(_bits(g.read_words("rows", 0, tot * C["ROWS"] * 4)), _bits(o.read("rows")[:tot * C["ROWS"] * 4])):
            return f"substep {sub} after frame {good_frames}: rows (prepare)"
        o.stage(2)
        g.debug_stage(2)
        if not np.array_equal(_bits(g.poses()), _bits(o.read("poses")[:pk.NB * 8])):
            return f"substep {sub} after frame {good_frames}: poses (solve)"
    return "no difference found when stepping stage by stage"


@pytest.mark.skipif(not NAMES, reason="packed reference scenes absent: run tests/golden/make_reference_scenes.py")
@pytest.mark.parametrize("name", NAMES)
def test_reference_scene_bit_exact(name, steel, oracle_lib, oracle_runs):
    pk = refscenes.load(name)
    g = Batch([pk])
    want = oracle_runs[name].result(timeout=1800)
    for k, w in enumerate(want):
        g.step(refscenes.EVERY)
        poses, vel, q, qd, _ = g.raw_state()
        st = g.stats()
        got = refscenes.snapshot(pk, poses, vel, np.zeros(0), [st["contacts"], st["colors"], st["max_pairs"], st["max_units"]])
        got["q"], got["qd"] = q, qd
        frame = refscenes.EVERY * (k + 1)
        for key in ("poses", "vel", "q", "qd"):
            if not np.array_equal(_bits(got[key]), _bits(w[key])):
                where = _first_difference(pk, frame - refscenes.EVERY, oracle_lib)
                pytest.fail(f"{name}: {key} differ at frame {frame}; first differing stage: {where}")
        assert got["stats"].tolist() == w["stats"].tolist(), f"{name}: stats differ at frame {frame}"
    g.close()
