"""The device-wide radix sort of large scenes' contacts (more padded keys than the block sort's
8192 shared-memory slots) against the oracle's canonical order, bit for bit: a 2200-box carpet
(8800 plane contacts) with the contact capacity 12000 (not a power of two), alone and in a batch
with a small scene and a second large scene (10000 contacts)."""
import numpy as np
import pytest

from steel_webgpu_b200 import pack
from steel_webgpu_b200.sim import Batch, auto_caps
from tests import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _carpet(n, seed):
    sc = scenes.box_carpet(n=n, seed=seed)
    caps = auto_caps(sc)
    caps.update(MAXC=12000, MAXU=12000)
    return pack(sc, caps=caps)


def _check_sorted(g, i, pk, o):
    o.collide()
    cnt = o.read("collide_counts", np.uint32)
    nc = min(int(cnt[1]), pk.C["MAXC"])
    rec, smu = g.contacts(i)
    oc = o.read("contacts")
    assert rec.shape[0] == nc
    assert np.array_equal(_bits(rec.reshape(-1)), _bits(oc[:nc * 20])), "sorted contact records differ"
    assert np.array_equal(_bits(smu.reshape(-1)), _bits(oc[pk.C["MAXC"] * 20:pk.C["MAXC"] * 20 + nc * 4]))
    return nc


def test_radix_sort_large_scene_alone(steel, oracle_lib):
    pk = _carpet(2200, 67)
    assert pk.C["MAXC"] == 12000
    g = Batch([pk])
    o = oracle_lib.OracleSim(pk)
    g.collide()
    assert _check_sorted(g, 0, pk, o) > 8192
    g.step(3)
    o.step(3)
    assert np.array_equal(_bits(g.poses()), _bits(o.read("poses")[:pk.NB * 8]))
    g.collide()
    assert _check_sorted(g, 0, pk, o) > 8192


def test_radix_sort_two_large_scenes_and_a_small_one(steel, oracle_lib):
    pks = [_carpet(2200, 67), pack(scenes.boxes(24)), _carpet(2500, 71)]
    g = Batch(pks)
    orcs = [oracle_lib.OracleSim(pk) for pk in pks]
    g.collide()
    counts = [_check_sorted(g, i, pk, o) for i, (pk, o) in enumerate(zip(pks, orcs))]
    assert counts[0] > 8192 and counts[2] > 8192 and counts[1] < 8192, counts
    g.step(2)
    for i, (pk, o) in enumerate(zip(pks, orcs)):
        o.step(2)
        assert np.array_equal(_bits(g.poses(i)), _bits(o.read("poses")[:pk.NB * 8])), f"scene {i} differs"
