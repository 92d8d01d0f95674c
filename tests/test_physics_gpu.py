"""The known-answer scenes of the oracle's physics tests (tests/test_oracle_physics_cpu.py) on the
CUDA path: Coulomb sliding on tilted gravity (along an axis and along the diagonal), a restitution
bounce, an inelastic collision in zero gravity, a free asymmetric spin without damping, and a
floating articulated chain set spinning in zero gravity. Poses and velocities match the oracle bit
for bit over the whole run, so the laws those tests check hold on the GPU as they do there."""
import math

import numpy as np
import pytest

from steel_webgpu_b200 import SceneBuilder, pack
from steel_webgpu_b200.sim import Batch

pytestmark = pytest.mark.gpu
G = 9.81


def _incline(gx, gy, mu):
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(gx, gy, -math.sqrt(G * G - gx * gx - gy * gy)))
    b.add_ground_plane(mu=mu)
    body = b.add_body(xform=[0.0, 0.0, 0.1, 0, 0, 0, 1])
    b.add_shape_box(body, hx=0.2, hy=0.15, hz=0.1, mu=mu)
    return b.finalize()


def _bounce(e):
    b = SceneBuilder(fps=240, gravity=(0.0, 0.0, -G))
    b.add_ground_plane(restitution=e)
    ball = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1])
    b.add_shape_sphere(ball, radius=0.1, restitution=e)
    return b.finalize()


def _collision():
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    a = b.add_body(xform=[-0.5, 0.0, 1.0, 0, 0, 0, 1], twist=(1.0, 0.0, 0.0, 0, 0, 0))
    b.add_shape_box(a, hx=0.1, hy=0.1, hz=0.1, restitution=0.0)
    c = b.add_body(xform=[0.5, 0.0, 1.0, 0, 0, 0, 1], twist=(-0.5, 0.0, 0.0, 0, 0, 0))
    b.add_shape_box(c, hx=0.15, hy=0.1, hz=0.1, restitution=0.0)
    return b.finalize()


def _spin():
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    body = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1], twist=(0.0, 0.0, 0.0, 0.3, 4.0, 0.2))
    b.add_shape_box(body, hx=0.3, hy=0.2, hz=0.1)
    sc = b.finalize()
    sc.json["bodies"]["angular_damping"] = [0.0]
    return sc


def _floating_chain():
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    base = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1], twist=(0.1, 0.0, 0.0, 0.5, 1.5, 2.0))
    b.add_shape_box(base, hx=0.2, hy=0.1, hz=0.05, mass=2.0)
    b.add_joint_free(base)
    parent, L = base, 0.3
    for k, axis in enumerate(([0, 1, 0], [1, 0, 0], [0, 0, 1])):
        link = b.add_body(xform=[0.2 + L * (k + 0.5), 0.0, 1.0, 0, 0, 0, 1])
        b.add_shape_capsule(link, radius=0.03, half_height=0.1, mass=0.5 + 0.5 * k)
        b.add_joint_revolute(parent, link, axis=axis,
                             parent_xform=[0.2 if k == 0 else L / 2, 0.0, 0.0, 0, 0, 0, 1],
                             child_xform=[-L / 2, 0.0, 0.0, 0, 0, 0, 1])
        parent = link
    sc = b.finalize()
    sc.json["bodies"]["angular_damping"] = [0.0] * 4
    return sc


SCENES = {
    "incline_slide": (lambda: _incline(G * math.sin(math.atan(0.8)), 0.0, 0.5), 240),
    "incline_diagonal": (lambda: _incline(*([G * math.sin(math.atan(0.9)) / math.sqrt(2.0)] * 2), 0.4), 240),
    "incline_stick": (lambda: _incline(G * math.sin(math.atan(0.55)), 0.0, 0.6), 240),
    "bounce": (lambda: _bounce(0.8), 300),
    "collision": (_collision, 240),
    "spin": (_spin, 480),
    "floating_chain": (_floating_chain, 240),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_known_answer_scenes_match_the_oracle(name, steel, oracle_lib):
    make, frames = SCENES[name]
    pk = pack(make())
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    for chunk in (frames // 2, frames - frames // 2):
        o.step(chunk)
        g.step(chunk)
        gp, gv, gq, gqd, _ = g.raw_state()
        assert np.array_equal(gp.view(np.uint32), o.read("poses")[:pk.NB * 8].view(np.uint32)), "poses differ"
        assert np.array_equal(gv.view(np.uint32), o.read("vel")[:pk.NB * 8].view(np.uint32)), "velocities differ"
        if pk.NQ:
            art = o.read("art")
            assert np.array_equal(gq.view(np.uint32), art[pk.C["A_Q"]:pk.C["A_Q"] + pk.NQ].view(np.uint32))
            assert np.array_equal(gqd.view(np.uint32), art[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND].view(np.uint32))
    g.close()
