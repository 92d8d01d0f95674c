"""Parity at the configurations' full sizes: the CUDA path against the CPU oracle, bit for bit, on
the 64-box plain scene over its full 1000 frames, the 8192-body pour, the 1024-quadruped +
64-chain articulation scene, and a sample of scenes inside the full 2048-scene uneven batch.

The oracle is slow at these sizes, so the large scenes are compared over their first frames
(where all collision and solver paths already run); the small scene over its whole run.
"""
import numpy as np
import pytest

from steel_webgpu_b200 import pack, synth
from steel_webgpu_b200.sim import Batch, auto_caps

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _pair_set(p):
    return {(int(min(a, b)), int(max(a, b))) for a, b in p}


def _same_state(g, o, pk, scene=0):
    assert np.array_equal(_bits(g.poses(scene)), _bits(o.read("poses")[:pk.NB * 8])), "poses differ"
    _, gv, gq, gqd, _ = g.raw_state(scene)
    assert np.array_equal(_bits(gv), _bits(o.read("vel")[:pk.NB * 8])), "velocities differ"
    if pk.NQ:
        art = o.read("art")
        assert np.array_equal(_bits(gq), _bits(art[pk.C["A_Q"]:pk.C["A_Q"] + pk.NQ])), "joint coordinates differ"
        assert np.array_equal(_bits(gqd), _bits(art[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND])), "joint speeds differ"


def test_boxes_64_full_run(steel, oracle_lib):
    """64 boxes dropped on a plane, 240 fps, 4 substeps, 12 iterations, all 1000 frames."""
    sc = synth.boxes_on_plane(64, seed=0)
    pk = pack(sc, caps=auto_caps(sc))
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    for chunk in range(4):
        o.step(250)
        g.step(250)
        _same_state(g, o, pk)


def test_convex_pour_8192(steel, oracle_lib):
    """8192 hulls, boxes and capsules poured into a 4 m bin: the initial candidate pair set
    (about 1e5 pairs) and the sorted contacts, then the state after 2 frames."""
    sc = synth.convex_pour(n=8192, seed=0)
    caps = auto_caps(sc)  # sized for piles of the uneven batch; the full pour needs about 12 pairs per shape
    caps.update(MAXP=1 << 18, MAXC=1 << 18, MAXU=1 << 18, UH=1 << 18, WH=1 << 19, AH=1 << 18)
    pk = pack(sc, caps=caps)
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    o.collide()
    g.collide()
    cnt = o.read("collide_counts", np.uint32)
    assert cnt[0] > 50000 and cnt[0] <= pk.C["MAXP"]
    op = o.read("pairs", np.uint32)[:cnt[0] * 2].reshape(-1, 2)
    assert _pair_set(g.pairs()) == _pair_set(op)
    rec, _ = g.contacts()
    assert rec.shape[0] == min(int(cnt[1]), pk.C["MAXC"])
    assert np.array_equal(_bits(rec.reshape(-1)), _bits(o.read("contacts")[:rec.shape[0] * 20]))
    o.step(2)
    g.step(2)
    _same_state(g, o, pk)
    assert g.stats()["overflow"] == []


def test_quadrupeds_1024_and_chains(steel, oracle_lib):
    """1024 PD-driven quadrupeds (13 links, 12 revolute joints each) and 64 serial 40-link chains
    with link mass ratios up to 1e3, 500 fps: state after 1 frame (4 substeps)."""
    sc = synth.quadrupeds(n_quad=1024, n_chains=64, chain_links=40, seed=0)
    pk = pack(sc, caps=auto_caps(sc))
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    o.step(1)
    g.step(1)
    _same_state(g, o, pk)


def test_uneven_batch_2048_sample(steel, oracle_lib):
    """The 2048-scene uneven batch of the bench (8-512 bodies and a 2-40 link chain per scene)
    stepped as one batch for 2 frames: a sample of its scenes, the largest included, matches each
    scene stepped alone by the oracle."""
    import bench
    pks = bench.build_workload("uneven_batch_2048", 0)
    g = Batch(pks)
    g.step(2)
    largest = int(np.argmax([pk.NB for pk in pks]))
    for i in sorted({0, 1, 777, 1500, 2047, largest}):
        o = oracle_lib.OracleSim(pks[i])
        o.step(2)
        _same_state(g, o, pks[i], scene=i)
