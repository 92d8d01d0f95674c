"""The user-control and readback surface through the C ABI against the oracle fed the same writes.

- setJointTarget / setJointForce / setBodyWrench / setBodyPose / setBodyTwist (sim.js:716-785):
  the GPU runs them through steel_set_*; the oracle gets the same words written into its art,
  poses and vel buffers, as the reference's queue.writeBuffer calls do, and its user-target flag
  (sim.js:720, :633). Poses, velocities and joint state must then agree bit for bit.
- Joint targets resampled every 50 frames through steel_step_io for a batch (the articulation
  workload's control loop), against the oracle given the same targets.
- Sim.state() in Newton layout (sim.js:732-763) against a restatement of that conversion applied
  to the oracle's raw buffers.
- Failure paths: a capacity overflow is reported in the stats, not as an error (sim.js:826-828);
  a shared-memory copy wait that runs out returns STEEL_E_TIMEOUT and leaves the context usable.
"""
import ctypes

import numpy as np
import pytest

from steel_webgpu_b200 import _lib, pack, synth
from steel_webgpu_b200.builder import JT
from steel_webgpu_b200.packer import LB, L_V
from steel_webgpu_b200.sim import Batch, Sim
from tests import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _assert_same_state(batch, o, pk, scene=0, what=""):
    nb = pk.NB
    gp, gv, gq, gqd, _ = batch.raw_state(scene)
    assert np.array_equal(_bits(gp), _bits(o.read("poses")[:nb * 8])), f"poses differ {what}"
    assert np.array_equal(_bits(gv), _bits(o.read("vel")[:nb * 8])), f"velocities differ {what}"
    oa = o.read("art")
    assert np.array_equal(_bits(gq), _bits(oa[pk.C["A_Q"]:pk.C["A_Q"] + pk.NQ])), f"joint coordinates differ {what}"
    assert np.array_equal(_bits(gqd), _bits(oa[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND])), f"joint velocities differ {what}"


def _newton_state(scene_json, pk, poses, vel, art):
    """sim.js:732-763 restated on the oracle's buffers: link COM twists replace the body velocity of
    articulated bodies, body origins are COM minus the rotated COM offset (in double, as JS does),
    joint coordinates come through the Newton -> port maps, and free joints outside articulations
    mirror their body."""
    J = scene_json["joints"]
    NB = pk.NB
    A_Q, A_QD, A_LINK = pk.C["A_Q"], pk.C["A_QD"], pk.C["A_LINK"]
    vel = np.array(vel[:NB * 8], dtype=np.float32)
    for l, link in enumerate(pk.links):
        o = A_LINK + l * LB + L_V
        w, v = art[o:o + 3], art[o + 3:o + 6]
        vel[link["body"] * 8:link["body"] * 8 + 8] = [v[0], v[1], v[2], 0, w[0], w[1], w[2], 0]
    body_q = np.zeros(NB * 7, dtype=np.float32)
    body_qd = np.zeros(NB * 6, dtype=np.float32)
    com = scene_json["bodies"]["com"]
    for b in range(NB):
        x, y, z, w = (float(t) for t in poses[b * 8 + 4:b * 8 + 8])
        c = [float(t) for t in com[b]]
        dot2 = 2 * (x * c[0] + y * c[1] + z * c[2])
        s2 = w * w - (x * x + y * y + z * z)
        cr = (y * c[2] - z * c[1], z * c[0] - x * c[2], x * c[1] - y * c[0])
        r = [dot2 * q + s2 * c[k] + 2 * w * cr[k] for k, q in enumerate((x, y, z))]
        body_q[b * 7:b * 7 + 7] = [float(poses[b * 8 + k]) - r[k] for k in range(3)] + [x, y, z, w]
        body_qd[b * 6:b * 6 + 6] = [vel[b * 8 + k] for k in (0, 1, 2, 4, 5, 6)]
    joint_q = np.array(J["q"], dtype=np.float32)
    joint_qd = np.zeros(J["qd_start"][-1], dtype=np.float32)
    for nq, q in pk.q_map.items():
        joint_q[nq] = art[A_Q + q]
    for nd, d in pk.dof_map.items():
        joint_qd[nd] = art[A_QD + d]
    for j, t in enumerate(J["type"]):
        if t not in (JT["FREE"], JT["DISTANCE"]) or J["q_start"][j] in pk.q_map:
            continue
        b = J["child"][j]
        joint_q[J["q_start"][j]:J["q_start"][j] + 7] = body_q[b * 7:b * 7 + 7]
        joint_qd[J["qd_start"][j]:J["qd_start"][j] + 6] = body_qd[b * 6:b * 6 + 6]
    return dict(bodyQ=body_q, bodyQd=body_qd, jointQ=joint_q, jointQd=joint_qd)


def test_setters_and_state_match_oracle(steel, oracle_lib):
    scene = scenes.controlled()
    sim = Sim(scene)
    pk = sim.packed
    C = pk.C
    o = oracle_lib.OracleSim(pk)
    linked = {link["body"] for link in pk.links}
    free = [b for b in range(pk.NB) if b not in linked]
    assert len(free) >= 4 and pk.ND >= 12
    dofs = sorted(pk.dof_map)
    sim.step(10)
    o.step(10)
    _assert_same_state(sim._batch, o, pk, what="before any write")

    # Joint targets (a policy's action vector over consecutive Newton dofs) and one joint force.
    first = dofs[0]
    pos = np.float32(np.linspace(-0.4, 0.4, 8))
    vel = np.float32(np.linspace(0.5, -0.5, 8))
    sim.setJointTargets(pos, vel, first=first)
    for k in range(8):
        d = pk.dof_map[first + k]
        o.write("art", C["A_TGT"] + d, [pos[k]])
        o.write("art", C["A_TGTV"] + d, [vel[k]])
    oracle_lib.lib().oracle_set_user_targets(o.h, 1)
    nd_force = dofs[-1]
    sim.setJointForce(nd_force, 0.75)
    o.write("art", C["A_JF"] + pk.dof_map[nd_force], [0.75])
    # A wrench on a resting box, held for the next frames.
    f, t = [30.0, -5.0, 20.0], [0.0, 0.0, 2.5]
    sim.setBodyWrench(free[0], f, t)
    o.write("art", C["A_BF"] + free[0] * 8, f + [0.0] + t + [0.0])
    sim.step(20)
    o.step(20)
    _assert_same_state(sim._batch, o, pk, what="after targets, joint force and wrench")

    # Place the airborne box and prescribe a resting box's twist.
    com, quat = [-2.2, -0.9, 1.2], [0.0, 0.0, float(np.sin(0.3)), float(np.cos(0.3))]
    sim.setBodyPose(free[3], com, quat)
    o.write("poses", free[3] * 8, com + [0.0] + quat)
    tw = [0.4, 0.0, 1.5, 0.0, 0.0, 3.0]
    sim.setBodyTwist(free[1], tw)
    o.write("vel", free[1] * 8, tw[:3] + [0.0] + tw[3:] + [0.0])
    sim.step(30)
    o.step(30)
    _assert_same_state(sim._batch, o, pk, what="after pose and twist")

    # Newton-layout state: the Python Sim's conversion against the restatement on oracle buffers.
    got = sim.state()
    want = _newton_state(scene.json, pk, o.read("poses"), o.read("vel"), o.read("art"))
    for k in ("bodyQ", "bodyQd", "jointQ", "jointQd"):
        assert got[k].shape == want[k].shape, k
        assert np.array_equal(_bits(got[k]), _bits(want[k])), f"state()[{k}] differs"
    sim.destroy()


def test_step_io_targets_resampled_every_50_frames(steel, oracle_lib):
    """Two scenes of quadrupeds and a chain in one batch; every 50 frames new targets for every
    dof go in through steel_step_io and poses come out; the oracle gets the same targets."""
    pks = [pack(synth.quadrupeds(n_quad=4, n_chains=1, chain_links=10, seed=s, fps=500)) for s in (3, 4)]
    g = Batch(pks)
    orcs = [oracle_lib.OracleSim(pk) for pk in pks]
    rng = np.random.default_rng(50)
    nt = sum(pk.ND for pk in pks)
    poses = np.zeros(sum(pk.NB * 8 for pk in pks), dtype=np.float32)
    for block in range(4):
        tg = rng.uniform(-0.5, 0.5, nt).astype(np.float32)
        g.step_io(50, tg, poses)
        off_t = off_p = 0
        for pk, o in zip(pks, orcs):
            o.write("art", pk.C["A_TGT"], tg[off_t:off_t + pk.ND])
            oracle_lib.lib().oracle_set_user_targets(o.h, 1)
            o.step(50)
            assert np.array_equal(_bits(poses[off_p:off_p + pk.NB * 8]), _bits(o.read("poses")[:pk.NB * 8])), \
                f"poses differ after {50 * (block + 1)} frames"
            off_t += pk.ND
            off_p += pk.NB * 8
    for i, (pk, o) in enumerate(zip(pks, orcs)):
        _assert_same_state(g, o, pk, scene=i, what="at the end")


@pytest.mark.parametrize("which", ["pairs", "contacts"])
def test_capacity_overflow_is_reported_not_raised(which, steel, oracle_lib):
    """A tiny pair (or contact) capacity: work is dropped, the step does not fail, and the stats'
    overflow bits name the buffer that filled up, as the oracle's counters do."""
    caps = dict(MAXP=4096, MAXC=4096, MAXU=4096, UH=4096, WH=8192, AH=4096, MAXDENSE=64)
    if which == "pairs":
        caps["MAXP"] = 8
    else:
        caps.update(MAXC=16, MAXU=16, UH=16, WH=64, AH=16)
    pk = pack(scenes.boxes(32), caps=caps)
    g = Batch([pk])
    o = oracle_lib.OracleSim(pk)
    g.step(40)
    g.sync()
    o.step(40)
    st = g.stats()
    ost = o.read("stats", np.uint32)
    assert which in st["overflow"], st
    assert (ost[4] >= caps["MAXP"]) if which == "pairs" else (ost[1] >= caps["MAXC"])
    assert np.isfinite(g.poses()).all()


def test_wait_timeout_is_reported_and_context_recovers(steel, oracle_lib):
    """A wait limit of 0 makes the staged link copy's bounded wait run out: the step reports
    STEEL_E_TIMEOUT (the kernel drained its copy and skipped the scene); with the default limit
    back, a reset replays the scene bit for bit against the oracle."""
    pk = pack(scenes.articulated())
    g = Batch([pk])
    L = _lib.load()
    _lib.check(L.steel_debug_set_wait_limit(g.h, 0))
    g.step(1)
    with pytest.raises(_lib.SteelError) as e:
        g.sync()
    assert e.value.code == 7, str(e.value)
    _lib.check(L.steel_debug_set_wait_limit(g.h, 16777216))
    g.reset()
    o = oracle_lib.OracleSim(pk)
    g.step(20)
    o.step(20)
    g.sync()
    _assert_same_state(g, o, pk, what="after the timeout and reset")


def test_pose_export_device_to_device(steel):
    """steel_copy_poses_device (the pose bridge's GPU-to-GPU copy) on a caller's stream gives the
    same records as the host readback, for every scene of a batch."""
    import torch
    torch.cuda.init()
    pks = [pack(s) for s in scenes.small_batch(n=4)]
    g = Batch(pks)
    g.step(12)
    L = _lib.load()
    side = torch.cuda.Stream()
    for i, pk in enumerate(pks):
        dst = torch.full((pk.NB * 8,), float("nan"), dtype=torch.float32, device="cuda:0")
        _lib.check(L.steel_copy_poses_device(g.h, i, ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(side.cuda_stream)))
        side.synchronize()
        assert np.array_equal(_bits(dst.cpu().numpy()), _bits(g.poses(i))), f"scene {i}"
    host = np.zeros(8, dtype=np.float32)
    assert L.steel_copy_poses_device(g.h, 0, ctypes.c_void_p(host.ctypes.data), None) == 1
