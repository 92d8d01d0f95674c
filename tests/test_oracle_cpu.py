"""CPU checks of the oracle: known physical answers, its sin/cos/atan2, its committed fixtures, and
the scene loader and packer on the reference's own scene folders (when they are on disk).

The reference has no golden vectors for this path (parity unpinned), so these tests pin the oracle
by analytic cases and by fixtures it produced earlier (tests/golden/make_golden.py).
"""
import math
import os

import numpy as np
import pytest

from steel_webgpu_b200 import SceneBuilder, pack
from tests import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_fixtures.npz")
# The reference's assets/scenes folder when it is checked out (STEEL_REFERENCE_SCENES); otherwise
# the packed copies that tests/golden/make_reference_scenes.py wrote.
REF_SCENES = os.environ.get("STEEL_REFERENCE_SCENES", "")


def test_trig_accuracy(oracle_lib):
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-10, 10, 100000), rng.uniform(-1e4, 1e4, 20000)]).astype(np.float32)
    s, c = oracle_lib.trig(x)
    xs = x.astype(np.float64)
    # Within one float ulp of the correctly rounded value.
    for got, ref in ((s, np.sin(xs)), (c, np.cos(xs))):
        ulp = np.abs(got.view(np.int32).astype(np.int64) - ref.astype(np.float32).view(np.int32).astype(np.int64))
        assert ulp.max() <= 1
    y = rng.uniform(-5, 5, 100000).astype(np.float32)
    z = rng.uniform(-5, 5, 100000).astype(np.float32)
    a = oracle_lib.atan2(y, z)
    ref = np.arctan2(y.astype(np.float64), z.astype(np.float64)).astype(np.float32)
    assert np.abs(a.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64)).max() <= 1
    assert oracle_lib.atan2(np.float32([0.0]), np.float32([-1.0]))[0] == np.float32(math.pi)


def test_free_fall_matches_semi_implicit_euler(oracle_lib):
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane()
    body = b.add_body(xform=[0.0, 0.0, 5.0, 0, 0, 0, 1])
    b.add_shape_box(body, hx=0.1, hy=0.1, hz=0.1)
    pk = pack(b.finalize())
    o = oracle_lib.OracleSim(pk)
    frames, substeps = 30, pk.params["substeps"]
    o.step(frames)
    dt = np.float32(1.0 / (240 * substeps))
    g = np.float32(-9.81)
    v, z = np.float32(0.0), np.float32(5.0)
    for _ in range(frames * substeps):
        v = np.float32(v + g * dt)
        z = np.float32(z + v * dt)
    np.testing.assert_allclose(o.body_poses()[0, 2], z, rtol=1e-6)
    np.testing.assert_allclose(o.read("vel")[2], v, rtol=1e-5)


def test_box_rests_on_plane(oracle_lib):
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.6)
    body = b.add_body(xform=[0.0, 0.0, 0.1, 0, 0, 0, 1])
    b.add_shape_box(body, hx=0.2, hy=0.15, hz=0.1, mu=0.6)
    o = oracle_lib.OracleSim(pack(b.finalize()))
    o.step(240)
    pose = o.body_poses()[0]
    vel = o.read("vel")[:8]
    assert abs(pose[2] - 0.1) < 2e-3
    assert abs(pose[0]) < 1e-4 and abs(pose[1]) < 1e-4
    assert np.abs(vel[[0, 1, 2, 4, 5, 6]]).max() < 1e-2


def test_pendulum_small_angle_period(oracle_lib):
    r, d = 0.05, 0.5
    b = SceneBuilder(fps=240)
    bob = b.add_body(xform=[0.0, 0.0, 2.0 - d, 0, 0, 0, 1])
    b.add_shape_sphere(bob, radius=r)
    b.add_joint_revolute(-1, bob, axis=[0, 1, 0], parent_xform=[0.0, 0.0, 2.0, 0, 0, 0, 1],
                         child_xform=[0.0, 0.0, d, 0, 0, 0, 1], q=[0.05])
    pk = pack(b.finalize())
    o = oracle_lib.OracleSim(pk)
    qs = []
    for _ in range(720):
        o.step(1)
        qs.append(o.read("art")[pk.C["A_Q"]])
    q = np.array(qs)
    t = (np.arange(len(q)) + 1) / 240.0
    cross = [t[i] - q[i] * (t[i + 1] - t[i]) / (q[i + 1] - q[i]) for i in range(len(q) - 1) if q[i] * q[i + 1] < 0]
    period = 2.0 * float(np.mean(np.diff(cross)))
    expected = 2.0 * math.pi * math.sqrt((0.4 * r * r + d * d) / (9.81 * d))
    assert len(cross) >= 4
    assert abs(period - expected) / expected < 0.01


def _fixture_values(oracle_lib):
    from tests.golden.make_golden import fixture_values
    return fixture_values(oracle_lib)


def test_oracle_matches_committed_fixtures(oracle_lib):
    gold = np.load(GOLDEN)
    now = _fixture_values(oracle_lib)
    assert sorted(now) == sorted(gold.files)
    for k in gold.files:
        a, b = np.ascontiguousarray(gold[k]), np.ascontiguousarray(now[k])
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"fixture {k} changed"


def test_longest_first_color_order(oracle_lib):
    """propagation_color_order "longest_first": rows are colored by row count first, so a scene
    whose points carry 1, 3 and 6 rows steps to a different (finite) state than in contact order."""
    def run(opts):
        pk = pack(scenes.spin_roll(), opts=opts)
        o = oracle_lib.OracleSim(pk)
        o.step(30)
        return pk, o.body_poses()

    pk, p_lf = run({"solver": {"propagation_color_order": "longest_first"}})
    _, p_co = run(None)
    assert pk.C["LONGEST_FIRST"] == 1
    assert np.isfinite(p_lf).all()
    assert not np.array_equal(p_lf, p_co)


def _reference_scenes_packed():
    from tests import refscenes
    if REF_SCENES and os.path.isdir(REF_SCENES):
        from steel_webgpu_b200.builder import load_scene
        names = sorted(d for d in os.listdir(REF_SCENES) if os.path.exists(os.path.join(REF_SCENES, d, "scene.json")))
        return [(n, pack(load_scene(os.path.join(REF_SCENES, n)))) for n in names]
    return [(n, refscenes.load(n)) for n in refscenes.names()]


@pytest.mark.skipif(not (REF_SCENES and os.path.isdir(REF_SCENES)) and not os.path.isdir(
    os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "_ref")),
                    reason="neither the reference scene folders nor their packed copies are on disk")
def test_reference_scenes_load_and_pack(oracle_lib):
    packed = _reference_scenes_packed()
    assert len(packed) >= 40
    for name, pk in packed:
        assert pk.statF.size == pk.C["LEN_STATF4"] * 4 and pk.statU.size == pk.C["LEN_STATU"], name
    for name, pk in packed:
        o = oracle_lib.OracleSim(pk)
        o.step(5)
        assert np.isfinite(o.body_poses()).all(), name


def test_joint_velocity_limits_hold(oracle_lib):
    def peak(opts):
        pk = pack(scenes.vel_limited(), opts=opts)
        o = oracle_lib.OracleSim(pk)
        m = 0.0
        for _ in range(120):
            o.step(1)
            m = max(m, float(np.abs(o.read("art")[pk.C["A_QD"]:pk.C["A_QD"] + 10]).max()))
        return pk.C["VLIM_ON"], m
    on, limited = peak(None)
    off, free = peak({"solver": {"enable_joint_velocity_limits": False}})
    assert on == 1 and off == 0
    assert limited < 2.05
    assert free > 2.5


def _chain_qdd_error(oracle_lib, height, n_links, ratio, fp64_option, seeds=3):
    """Worst max |qdd - qdd64| / max |qdd64| over seeded serial revolute chains (link masses
    log-uniform over `ratio`, random joint angles, qd = 0): the oracle's articulated-body pass (one
    prepare) against the float64 joint-space dynamics of tests/fp64_aba.py."""
    from steel_webgpu_b200 import synth
    from tests.fp64_aba import qdd_fp64
    worst = 0.0
    for seed in range(seeds):
        b = SceneBuilder(fps=240)
        synth._add_chain(b, np.random.default_rng(seed), [0.0, 0.0, height], n_links, ratio_max=ratio)
        pk = pack(b.finalize(), opts={"solver": {"articulation_fp64": fp64_option}})
        C = pk.C
        assert C["ART_F64"] == (1 if fp64_option else 0)
        pk.art[C["A_Q"]:C["A_Q"] + pk.NQ] = np.random.default_rng(100 + seed).uniform(-0.6, 0.6, pk.NQ)
        dt = float(np.float32(1.0 / (pk.params["fps"] * pk.params["substeps"])))
        o = oracle_lib.OracleSim(pk)
        o.stage(0)
        o.stage(1)
        qdd = o.read("art")[C["A_QDH"]:C["A_QDH"] + pk.ND].astype(np.float64) / dt
        qdd64 = qdd_fp64(pk, dt)
        worst = max(worst, float(np.abs(qdd - qdd64).max() / np.abs(qdd64).max()))
    return worst


@pytest.mark.parametrize("height,n_links,bound", [(0.0, 2, 1e-6), (0.0, 40, 2e-5), (5.0, 40, 2e-5)])
def test_articulation_fp32_error_against_fp64(oracle_lib, height, n_links, bound):
    """FP32 pass (the reference's precision) on chains with a 10^3 mass ratio. World-frame link
    positions are FP32, so the error grows with the chain's distance from the origin; the GPU path
    is bit-identical to the oracle here."""
    assert _chain_qdd_error(oracle_lib, height, n_links, 1e3, False) < bound


def test_articulation_fp64_option_error(oracle_lib):
    """The FP64 articulated-inertia option (D = S^T I^A S, its inverse and the inertia accumulation
    toward the root in double) on 40-link chains with a 10^5 mass ratio: at least 3x below the FP32
    pass's error against FP64, and below 4e-6."""
    e32 = _chain_qdd_error(oracle_lib, 0.0, 40, 1e5, False)
    e64 = _chain_qdd_error(oracle_lib, 0.0, 40, 1e5, True)
    assert e64 < 4e-6
    assert e32 > 3.0 * e64


@pytest.mark.parametrize("opts", [dict(), dict(cone="pyramidal", creep=0.01)])
def test_articulated_rolling_and_spin_friction(oracle_lib, opts):
    """enable_torsional_rolling_friction: a dumbbell rolling across its bar at 1 m/s slows down and
    one spinning flat at 6 rad/s stops, while without the option the rolling one keeps its speed."""
    from tests import scenes

    def run(on):
        sc = scenes.ang_art(**opts)
        sc.json["solver"]["enable_torsional_rolling_friction"] = on
        pk = pack(sc)
        o = oracle_lib.OracleSim(pk)
        o.step(60)
        qd60 = o.read("art")[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND].copy()
        o.step(90)
        qd150 = o.read("art")[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND].copy()
        return qd60, qd150, o.body_poses()

    on60, on150, p_on = run(True)
    off60, off150, _ = run(False)
    assert np.isfinite(p_on).all()
    assert abs(off60[7]) > 0.99                     # rolling dumbbell, no angular friction: ~1 m/s
    assert 0.2 < abs(on60[7]) < 0.8                 # rolling resistance mu_r N over 0.25 s
    assert np.linalg.norm(off150[3:6]) > 3.0        # the spinning one keeps spinning without it
    assert np.linalg.norm(on150[3:6]) < 0.1         # and stops with it


def test_mimic_joints_follow_their_reference(oracle_lib):
    """set_joint_mimic: the second arm holds q2 = 0.1 - q1 and the second finger q4 = -q3 while the
    driven joints move (mimic rows in the dense pass)."""
    from tests import scenes
    pk = pack(scenes.mimic_arms())
    assert pk.C["NMIMIC"] == 2
    o = oracle_lib.OracleSim(pk)
    o.step(60)
    q = o.read("art")[pk.C["A_Q"]:pk.C["A_Q"] + pk.NQ]
    assert q[0] > 0.2                       # the driven arm has moved toward its target
    assert abs(q[1] - (0.1 - q[0])) < 2e-3
    assert abs(q[2]) > 0.01 and abs(q[3] + q[2]) < 2e-3
