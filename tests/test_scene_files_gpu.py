"""Scenes created from their own files through the C ABI (steel_scene_create: scene.json text and
scene.bin bytes, packed in C++) step exactly like the same scenes packed in Python, and
steel_state returns Sim.state()'s Newton layout (sim.js:732-763) bit for bit."""
import ctypes
import json

import numpy as np
import pytest

from steel_webgpu_b200 import _lib, pack
from steel_webgpu_b200.sim import Batch, Sim, _Context
from tests import refscenes, scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _create(text: bytes, bn: bytes, opts=None):
    L = _lib.load()
    h = ctypes.c_void_p()
    b = ctypes.create_string_buffer(bn, len(bn))
    _lib.check(L.steel_scene_create(_Context.get(0), text, len(text), ctypes.cast(b, ctypes.c_void_p), len(bn),
                                    json.dumps(opts).encode() if opts else None, ctypes.byref(h)))
    return h.value


def _poses(h, nb):
    out = np.zeros(nb * 8, dtype=np.float32)
    _lib.check(_lib.load().steel_read_poses(h, 0, out.ctypes.data))
    return out


def _state(h):
    L = _lib.load()
    info = _lib.NewtonInfo()
    _lib.check(L.steel_newton_info(h, 0, ctypes.byref(info)))
    out = [np.zeros(max(n, 1), dtype=np.float32) for n in (info.bodies * 7, info.bodies * 6, info.joint_coords,
                                                          info.joint_dofs)]
    _lib.check(L.steel_state(h, 0, *[a.ctypes.data for a in out]))
    return dict(zip(("bodyQ", "bodyQd", "jointQ", "jointQd"), [out[0], out[1], out[2][:info.joint_coords],
                                                                out[3][:info.joint_dofs]]))


@pytest.mark.parametrize("name", [n for n in ("ragdoll", "dominoes", "linkages", "toy_piano", "cereal")
                                  if n in refscenes.names()] or ["absent"])
def test_scene_files_step_like_the_python_packed_scene(name, steel):
    if name == "absent":
        pytest.skip("packed reference scenes absent")
    text, bn = refscenes.files(name)
    pk = refscenes.load(name)
    h = _create(text, bn)
    g = Batch([pk])
    L = _lib.load()
    _lib.check(L.steel_step(h, 60))
    g.step(60)
    assert np.array_equal(_bits(_poses(h, pk.NB)), _bits(g.poses())), name
    L.steel_batch_destroy(h)


def test_steel_state_matches_the_python_state(steel):
    sc = scenes.controlled()
    sim = Sim(sc)
    h = _create(json.dumps(sc.json).encode(), sc.bin)
    L = _lib.load()
    sim.step(25)
    _lib.check(L.steel_step(h, 25))
    want = sim.state()
    got = _state(h)
    for k in want:
        assert np.array_equal(_bits(got[k]), _bits(want[k])), k
    # Newton dof -> port dof, and the reference's error for a dof outside the articulations.
    port = ctypes.c_uint32()
    nd = sorted(sim.packed.dof_map)[3]
    _lib.check(L.steel_newton_dof(h, 0, nd, ctypes.byref(port)))
    assert port.value == sim.packed.dof_map[nd]
    free_dof = next(d for d in range(len(sc.json["joints"]["axis"]) + 20) if d not in sim.packed.dof_map)
    assert L.steel_newton_dof(h, 0, free_dof, ctypes.byref(port)) == 1
    assert b"is not simulated as an articulation dof" in L.steel_last_error()
    L.steel_batch_destroy(h)
    sim.destroy()


def test_batch_from_files_matches_packed_batch(steel):
    """Several scenes created from their files in one batch (steel_batch_create_files) step like the
    same scenes packed in Python, options included."""
    scs = [scenes.boxes(20), scenes.articulated()]
    opts = [None, {"solver": {"drive_mode": "rows"}}]
    fb = Batch.from_files([(json.dumps(sc.json).encode(), sc.bin, o) for sc, o in zip(scs, opts)])
    pb = Batch([pack(sc, opts=o) for sc, o in zip(scs, opts)])
    L = _lib.load()
    _lib.check(L.steel_step(fb.h, 15))
    pb.step(15)
    for i, sc in enumerate(scs):
        nb = sc.json["bodies"]["count"]
        assert np.array_equal(_bits(_poses_of(fb.h, i, nb)), _bits(pb.poses(i))), f"scene {i}"
    fb.close()


def _poses_of(h, scene, nb):
    out = np.zeros(nb * 8, dtype=np.float32)
    _lib.check(_lib.load().steel_read_poses(h, scene, out.ctypes.data))
    return out
