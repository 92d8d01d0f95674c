"""The library's C++ packer (steel_pack / steel_scene_create; Sim.build of sim.js:95-521 restated in
C++) against the Python packer the parity tests use, word for word: statF, statU, the initial
pose, velocity and articulation buffers, and every constant. On the builder's test scenes with the
solver options the GPU parity tests use, and on the reference's own scene folders (their packed
copies, when tests/golden/make_reference_scenes.py has written them). CPU only: packing needs no
device."""
import ctypes
import json

import numpy as np
import pytest

from steel_webgpu_b200 import _lib, pack
from tests import refscenes, scenes
from tests.test_parity_gpu import OPTS, SCENES


def _parse_constants(text: str) -> dict:
    out = {}
    for line in text.strip().splitlines():
        k, v = line.split("=", 1)
        out[k] = float(v)
    return out


def cpp_pack(json_text: bytes, bin_bytes: bytes, opts: dict | None = None):
    L = _lib.load()
    p = ctypes.c_void_p()
    b = ctypes.create_string_buffer(bin_bytes, len(bin_bytes))
    rc = L.steel_pack(json_text, len(json_text), ctypes.cast(b, ctypes.c_void_p), len(bin_bytes),
                      json.dumps(opts).encode() if opts else None, ctypes.byref(p))
    _lib.check(rc)
    d = _lib.SceneDesc()
    _lib.check(L.steel_packed_desc(p, ctypes.byref(d)))

    def arr(ptr, n, dt):
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(dt)), shape=(n,)).copy() if n else np.zeros(0)

    nb = None
    consts = _parse_constants(d.constants.decode())
    nb = int(consts["NB"])
    out = dict(C=consts, statF=arr(d.statF, d.statF_floats, ctypes.c_float),
               statU=arr(d.statU, d.statU_words, ctypes.c_uint32),
               body_pose=arr(d.body_pose, nb * 8, ctypes.c_float), body_vel=arr(d.body_vel, nb * 8, ctypes.c_float),
               art=arr(d.art, d.art_floats, ctypes.c_float))
    L.steel_packed_free(p)
    return out


def _compare(pk, got, what):
    want_c = _parse_constants(pk.constants_text())
    assert set(got["C"]) == set(want_c), f"{what}: constant keys differ: {set(got['C']) ^ set(want_c)}"
    bad = {k: (got["C"][k], want_c[k]) for k in want_c if got["C"][k] != want_c[k]}
    assert not bad, f"{what}: constants differ: {bad}"
    for k in ("statF", "body_pose", "body_vel", "art"):
        a = np.ascontiguousarray(getattr(pk, k), dtype=np.float32).view(np.uint32)
        b = np.ascontiguousarray(got[k], dtype=np.float32).view(np.uint32)
        assert a.shape == b.shape, f"{what}: {k} sizes {a.shape} vs {b.shape}"
        if not np.array_equal(a, b):
            i = int(np.flatnonzero(a != b)[0])
            pytest.fail(f"{what}: {k} differs first at word {i}: {a.view(np.float32)[i]} vs {b.view(np.float32)[i]}")
    assert np.array_equal(pk.statU, got["statU"]), f"{what}: statU differs"


@pytest.mark.parametrize("name", sorted(SCENES))
def test_cpp_packer_matches_python_on_test_scenes(name, steel):
    sc = SCENES[name]()
    opts = OPTS.get(name)
    _compare(pack(sc, opts=opts), cpp_pack(json.dumps(sc.json).encode(), sc.bin, opts), name)


def test_cpp_packer_capacities_and_options(steel):
    sc = scenes.controlled()
    caps = dict(MAXP=4096, MAXC=12000, MAXU=12000, UH=16384, WH=32768, AH=16384, MAXDENSE=1024)
    opts = {"substeps": 6, "iterations": 9, "solver": {"friction_mode": "bisection"}}
    _compare(pack(sc, opts=opts, caps=caps), cpp_pack(json.dumps(sc.json).encode(), sc.bin,
                                                      dict(opts, capacities=caps)), "controlled")


@pytest.mark.skipif(not refscenes.names(), reason="packed reference scenes absent")
@pytest.mark.parametrize("name", refscenes.names() or ["none"])
def test_cpp_packer_matches_python_on_reference_scenes(name, steel):
    text, bn = refscenes.files(name)
    _compare(refscenes.load(name), cpp_pack(text, bn), name)


def test_cpp_packer_errors(steel):
    L = _lib.load()
    p = ctypes.c_void_p()
    assert L.steel_pack(b"{not json", 9, None, 0, None, ctypes.byref(p)) == 1
    assert b"scene.json" in L.steel_last_error()
    sc = scenes.boxes(4)
    text = json.dumps(sc.json).encode()
    b = ctypes.create_string_buffer(sc.bin, len(sc.bin))
    rc = L.steel_pack(text, len(text), ctypes.cast(b, ctypes.c_void_p), len(sc.bin),
                      b'{"solver": {"friction_mode": "magic"}}', ctypes.byref(p))
    assert rc == 1 and b"friction_mode magic is not supported" in L.steel_last_error()


def test_cpp_packer_collision_worlds_and_groups(steel):
    """Shapes spread over worlds (-1 shared, 0, 1) and collision groups (0 none, positive, negative,
    -1 all): the filter bitset of sim.js:235-255 from the C++ packer equals the Python packer's."""
    from steel_webgpu_b200 import SceneBuilder
    rng = np.random.default_rng(4)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane()
    for i in range(60):
        body = b.add_body(xform=[0.3 * (i % 8), 0.3 * (i // 8), 0.5, 0, 0, 0, 1])
        b.add_shape_box(body, hx=0.1, hy=0.1, hz=0.1, world=int(rng.choice([-1, 0, 1])),
                        collisionGroup=int(rng.choice([-1, 0, 1, 2, -2, -3])))
    sc = b.finalize()
    pk = pack(sc)
    ns = pk.C["NS"]
    bits = pk.statU[pk.C["SU_FILTER"]:pk.C["SU_FILTER"] + (ns * ns + 31) // 32]
    assert 0 < int(np.unpackbits(bits.view(np.uint8)).sum()) < ns * ns  # some pairs filtered, not all
    _compare(pk, cpp_pack(json.dumps(sc.json).encode(), sc.bin), "worlds and groups")
