"""The oracle's all-FP64 instance (o_f64.h), the precision reference of the articulation
workload's report (tests/precision_c3.py), on the CPU."""
import numpy as np
import pytest

import precision_c3
import scenes
from oracle.oracle import OracleSim
from steel_webgpu_b200 import SceneBuilder
from steel_webgpu_b200.packer import pack


def _free_fall():
    b = SceneBuilder(fps=240)
    body = b.add_body(xform=[0.3, -0.2, 100.0, 0, 0, 0, 1])
    b.add_shape_box(body, hx=0.1, hy=0.1, hz=0.1)
    return pack(b.finalize())


def test_fp64_instance_integrates_free_fall_in_double():
    """One second of free fall (240 frames x 4 substeps of v += g dt, x += v dt): the FP64 instance
    lands on the double-precision recurrence (to the binary32 rounding of the read), the float
    instance drifts by tens of ulps in the velocity."""
    pk = _free_fall()
    dt = 1.0 / 240.0 / 4.0
    z, v = 100.0, 0.0
    for _ in range(960):
        v += -9.81 * dt
        z += v * dt
    got = {}
    for f64 in (False, True):
        o = OracleSim(pk, f64=f64)
        o.step(240)
        got[f64] = (float(o.body_poses()[0][2]), float(o.read("vel")[2]))
    ulp_v = float(np.spacing(np.float32(9.81)))
    assert got[True][1] == float(np.float32(v)), got
    assert abs(got[True][0] - z) <= float(np.spacing(np.float32(z))), got
    assert abs(got[False][1] - v) > 10 * ulp_v, got


def test_fp64_instance_keeps_the_state_words_and_indices():
    """Contacts, pairs and colors of a box pile are integer words the FP64 instance must carry
    unchanged: after one substep's collision stage its pair list and contact count equal the float
    instance's (the same inputs, rounding-level differences in the positions)."""
    pk = pack(scenes.boxes(24))
    a, b = OracleSim(pk), OracleSim(pk, f64=True)
    a.step(30)
    b.step(30)
    a.collide()
    b.collide()
    na, nb = a.read("collide_counts"), b.read("collide_counts")
    assert np.array_equal(na.view(np.uint32), nb.view(np.uint32))
    npairs = int(na.view(np.uint32)[0])
    assert npairs > 0
    assert np.array_equal(a.read("pairs", np.uint32)[:2 * npairs], b.read("pairs", np.uint32)[:2 * npairs])
    pa, pb = a.body_poses(), b.body_poses()
    assert np.allclose(pa, pb, rtol=0, atol=1e-4)


@pytest.mark.parametrize("frames", [60])
def test_precision_report_small(frames):
    """The report on 2 quadrupeds and one 40-link chain: every quantity's error against the FP64 run
    is above zero (the runs differ in precision) and below 1e-3 relative after a few frames."""
    rep = precision_c3.main(["--quads", "2", "--chains", "1", "--frames", str(frames)])
    for leg in ("fp32", "fp32+fp64 D^-1"):
        e10 = rep["errors"][leg][10]
        for group in ("quadrupeds", "chains"):
            for q in precision_c3.QUANTITIES:
                assert 0.0 < e10[group][q] < 1e-3, (leg, group, q, e10[group][q])


def test_pd_arm_fp32_within_tolerance_of_fp64_over_1000_frames():
    """A PD-held three-link arm settling under gravity (no contact, no chaos): the float run stays
    within 1e-5 relative of the all-FP64 run in poses and joint angles over 1000 frames."""
    ell = 0.3
    b = SceneBuilder(fps=240)
    parent = -1
    for k in range(3):
        body = b.add_body(xform=[0.0, 0.0, 2.0 - ell * (k + 0.5), 0, 0, 0, 1])
        b.add_shape_capsule(body, radius=0.02, half_height=0.1, mass=[1.0, 0.7, 0.4][k])
        b.add_joint_revolute(parent, body, axis=[0, 1, 0],
                             parent_xform=[0.0, 0.0, -ell / 2 if parent >= 0 else 2.0, 0, 0, 0, 1],
                             child_xform=[0.0, 0.0, ell / 2, 0, 0, 0, 1], targetKe=300.0, targetKd=20.0,
                             targetPos=[0.6, -0.4, 0.8][k])
        parent = body
    pk = pack(b.finalize())
    f32, f64 = OracleSim(pk), OracleSim(pk, f64=True)
    q0, nq = pk.C["A_Q"], pk.NQ
    for _ in range(10):
        f32.step(100)
        f64.step(100)
        pa, pb = (o.read("poses")[:pk.NB * 8].astype(np.float64) for o in (f32, f64))
        qa, qb = (o.read("art")[q0:q0 + nq].astype(np.float64) for o in (f32, f64))
        assert np.linalg.norm(pa - pb) / np.linalg.norm(pb) < 1e-5
        assert np.linalg.norm(qa - qb) / np.linalg.norm(qb) < 1e-5
