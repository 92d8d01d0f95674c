"""Known physical answers for the oracle (CPU): the laws the reference's contact solve is built to
satisfy, checked on small scenes where the answer is analytic.

- Coulomb friction (the fixed-normal rows with friction anchors, wgsl.js:2952-3011, 3033-3231): a
  box on a tilted-gravity plane sticks below the friction angle and slides above it with
  acceleration g (sin t - mu cos t), along the tangential part of gravity whatever its direction.
- Restitution (wgsl.js:1333-1337 and 2166-2173, a firing row targets e times the closing speed):
  the rebound speed of a sphere dropped on the plane is e times the impact speed.
- Momentum (equal and opposite row impulses): a perfectly inelastic head-on collision in zero
  gravity keeps the total momentum and ends at the common velocity p / (m1 + m2).
- Free rotation (the Cayley gyroscopic microsteps, wgsl.js:2543-2562): an asymmetric box spinning
  in zero gravity without damping keeps its angular momentum and kinetic energy, also about the
  unstable middle axis.
- Articulated dynamics (the articulated-body factorisation and propagation, artwgsl.js, whose link
  motion is (w, v_com) at each link's COM, artwgsl.js:1-6): a floating base with a three-link
  revolute chain in zero gravity, set moving through its joint speeds, keeps its linear and
  angular momentum up to the first-order error of the time step: the drift halves with the step.
- Joints (articulated-body dynamics with implicit PD drives in D, artwgsl.js:4-6; limit rows,
  wgsl.js:3404-3468; joint integration, wgsl.js:3797-3826): a PD-driven pendulum settles where the
  drive torque balances gravity, ke (q* - q) = m g d sin q; a revolute limit holds against a swing
  that would pass it; a prismatic slide along a tilted axis follows the semi-implicit Euler
  recurrence of g . axis exactly; a ball-joint conical pendulum started at the steady rate
  sqrt(g / (L cos t)) keeps its cone angle and that rate; a three-link arm held by PD drives
  comes to rest where each joint's drive and damping balance the gravity torque of the links below
  it, ke (q* - q) - kd qd + sum_j m_j g (x_j - x_joint) = 0.
"""
import math

import numpy as np
import pytest

from steel_webgpu_b200 import SceneBuilder, pack
from steel_webgpu_b200.packer import LB, L_V

G = 9.81


def _box_on_tilted_plane(oracle_lib, gx, gy, mu, frames):
    gz = -math.sqrt(G * G - gx * gx - gy * gy)
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(gx, gy, gz))
    b.add_ground_plane(mu=mu)
    body = b.add_body(xform=[0.0, 0.0, 0.1, 0, 0, 0, 1])
    b.add_shape_box(body, hx=0.2, hy=0.15, hz=0.1, mu=mu)
    o = oracle_lib.OracleSim(pack(b.finalize()))
    pos, vel = [], []
    for _ in range(frames):
        o.step(1)
        pos.append(o.body_poses()[0, :3].astype(np.float64))
        vel.append(o.read("vel")[:3].astype(np.float64))
    return np.array(pos), np.array(vel)


@pytest.mark.parametrize("tan_t,mu", [(0.3, 0.6), (0.55, 0.6)])
def test_incline_sticks_below_the_friction_angle(oracle_lib, tan_t, mu):
    t = math.atan(tan_t)
    pos, vel = _box_on_tilted_plane(oracle_lib, G * math.sin(t), 0.0, mu, 240)
    assert np.abs(pos[-1, :2]).max() < 1e-4
    assert np.abs(vel[-1]).max() < 1e-3


@pytest.mark.parametrize("tan_t,mu", [(1.0, 0.3), (0.8, 0.5), (0.7, 0.2)])
def test_incline_slides_with_coulomb_acceleration(oracle_lib, tan_t, mu):
    t = math.atan(tan_t)
    _, vel = _box_on_tilted_plane(oracle_lib, G * math.sin(t), 0.0, mu, 240)
    a = (vel[200, 0] - vel[100, 0]) / (100.0 / 240.0)
    expected = G * (math.sin(t) - mu * math.cos(t))
    assert abs(a - expected) / expected < 5e-3
    assert np.abs(vel[200, 1:]).max() < 1e-4


def test_sliding_follows_the_tangential_gravity(oracle_lib):
    """Gravity tilted along the diagonal of the plane: the box slides along that diagonal at the
    Coulomb rate (the friction cone is round, not a pyramid along the box's axes)."""
    t, mu = math.atan(0.9), 0.4
    s = G * math.sin(t) / math.sqrt(2.0)
    _, vel = _box_on_tilted_plane(oracle_lib, s, s, mu, 240)
    v = vel[200, :2]
    assert abs(v[0] - v[1]) / abs(v[0]) < 1e-3
    a = (np.linalg.norm(vel[200, :2]) - np.linalg.norm(vel[100, :2])) / (100.0 / 240.0)
    expected = G * (math.sin(t) - mu * math.cos(t))
    assert abs(a - expected) / expected < 5e-3


@pytest.mark.parametrize("e,tol", [(0.5, 1e-3), (0.8, 5e-3)])
def test_restitution_rebound_speed(oracle_lib, e, tol):
    b = SceneBuilder(fps=240, gravity=(0.0, 0.0, -G))
    b.add_ground_plane(restitution=e)
    ball = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1])
    b.add_shape_sphere(ball, radius=0.1, restitution=e)
    o = oracle_lib.OracleSim(pack(b.finalize()))
    vz = []
    for _ in range(300):
        o.step(1)
        vz.append(float(o.read("vel")[2]))
    vz = np.array(vz)
    k = int(np.argmax(vz > 0.0))  # first frame moving up
    assert k > 0
    assert abs(-vz[k] / vz[k - 1] - e) < tol * e


def test_inelastic_collision_keeps_momentum(oracle_lib):
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    a = b.add_body(xform=[-0.5, 0.0, 1.0, 0, 0, 0, 1], twist=(1.0, 0.0, 0.0, 0, 0, 0))
    b.add_shape_box(a, hx=0.1, hy=0.1, hz=0.1, restitution=0.0)
    c = b.add_body(xform=[0.5, 0.0, 1.0, 0, 0, 0, 1], twist=(-0.5, 0.0, 0.0, 0, 0, 0))
    b.add_shape_box(c, hx=0.15, hy=0.1, hz=0.1, restitution=0.0)
    o = oracle_lib.OracleSim(pack(b.finalize()))
    ma, mc = 1000.0 * 0.2 * 0.2 * 0.2, 1000.0 * 0.3 * 0.2 * 0.2
    p0 = ma * 1.0 - mc * 0.5
    o.step(240)
    v = o.read("vel")[:16].reshape(2, 8).astype(np.float64)
    p = ma * v[0, :3] + mc * v[1, :3]
    assert abs(p[0] - p0) / p0 < 1e-6 and np.abs(p[1:]).max() < 1e-6
    np.testing.assert_allclose(v[:, 0], p0 / (ma + mc), rtol=1e-3)  # they move together


def _qmat(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


@pytest.mark.parametrize("w0", [(0.3, 4.0, 0.2), (5.0, 0.1, 0.1), (0.05, 0.2, 6.0)])
def test_free_spin_keeps_angular_momentum_and_energy(oracle_lib, w0):
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    body = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1], twist=(0.0, 0.0, 0.0) + tuple(w0))
    b.add_shape_box(body, hx=0.3, hy=0.2, hz=0.1)
    sc = b.finalize()
    sc.json["bodies"]["angular_damping"] = [0.0]
    o = oracle_lib.OracleSim(pack(sc))
    m = 1000.0 * 0.6 * 0.4 * 0.2
    inertia = np.diag([m / 3 * (0.2 ** 2 + 0.1 ** 2), m / 3 * (0.3 ** 2 + 0.1 ** 2), m / 3 * (0.3 ** 2 + 0.2 ** 2)])
    L, E = [], []
    for _ in range(480):
        pose, vel = o.body_poses()[0], o.read("vel")[:8]
        R = _qmat(pose[4:8].astype(np.float64))
        w = vel[4:7].astype(np.float64)
        Iw = R @ inertia @ R.T
        L.append(Iw @ w)
        E.append(0.5 * w @ Iw @ w)
        o.step(1)
    L, E = np.array(L), np.array(E)
    assert np.abs(L - L[0]).max() / np.linalg.norm(L[0]) < 2e-3
    assert np.abs(E - E[0]).max() / E[0] < 2e-3
    assert np.array_equal(o.body_poses()[0, :3], np.float32([0.0, 0.0, 1.0]))  # no drift of the centre


def _floating_chain_drift(oracle_lib, fps, seconds=0.5):
    """Largest relative change of the total linear and angular momentum over `seconds`."""
    b = SceneBuilder(fps=fps, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    base = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1])
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
    pk = pack(sc)
    C = pk.C
    o = oracle_lib.OracleSim(pk)
    o.write("art", C["A_QD"], [0.1, 0.0, 0.0, 0.0, 0.0, 0.5, 2.0, -1.5, 3.0])  # free joint, then revolutes
    rec = pk.statF.reshape(-1, 4)[C["SF_BODY"]:C["SF_BODY"] + pk.NB * 8].astype(np.float64).reshape(pk.NB, 8, 4)
    mass = 1.0 / rec[:, 0, 0]
    inertia = rec[:, 2:5, :3]

    def momentum():
        poses, art = o.body_poses(), o.read("art")
        lin, ang = np.zeros(3), np.zeros(3)
        for l, link in enumerate(pk.links):
            bb = link["body"]
            o6 = C["A_LINK"] + l * LB + L_V
            w, v = art[o6:o6 + 3].astype(np.float64), art[o6 + 3:o6 + 6].astype(np.float64)
            c = poses[bb, :3].astype(np.float64)
            R = _qmat(poses[bb, 4:8].astype(np.float64))
            lin += mass[bb] * v
            ang += R @ inertia[bb] @ R.T @ w + mass[bb] * np.cross(c, v)
        return lin, ang

    o.step(1)  # the link motion follows the written joint speeds from the first step on
    l0, a0 = momentum()
    dl = da = 0.0
    for _ in range(int(seconds * fps)):
        o.step(1)
        lin, ang = momentum()
        dl = max(dl, np.linalg.norm(lin - l0) / np.linalg.norm(l0))
        da = max(da, np.linalg.norm(ang - a0) / np.linalg.norm(a0))
    return dl, da


def test_floating_chain_keeps_momentum_to_first_order(oracle_lib):
    d240 = _floating_chain_drift(oracle_lib, 240)
    d480 = _floating_chain_drift(oracle_lib, 480)
    assert max(d240) < 3e-3
    for coarse, fine in zip(d240, d480):
        assert 0.4 < fine / coarse < 0.6  # first order in the time step


def _pendulum(ke=0.0, kd=0.0, target=0.0, limits=None, m=None, d=0.5, r=0.05):
    b = SceneBuilder(fps=240)
    bob = b.add_body(xform=[0.0, 0.0, 2.0 - d, 0, 0, 0, 1])
    b.add_shape_sphere(bob, radius=r, **({} if m is None else {"mass": m}))
    lim = {} if limits is None else {"limitLower": limits[0], "limitUpper": limits[1]}
    b.add_joint_revolute(-1, bob, axis=[0, 1, 0], parent_xform=[0.0, 0.0, 2.0, 0, 0, 0, 1],
                         child_xform=[0.0, 0.0, d, 0, 0, 0, 1], targetKe=ke, targetKd=kd, targetPos=target, **lim)
    return pack(b.finalize())


@pytest.mark.parametrize("ke", [50.0, 200.0])
def test_pd_drive_settles_at_the_torque_balance(oracle_lib, ke):
    m, d, target = 2.0, 0.5, 0.5
    pk = _pendulum(ke=ke, kd=5.0, target=target, m=m, d=d)
    o = oracle_lib.OracleSim(pk)
    o.step(1200)
    art = o.read("art")
    f = lambda t: ke * (target - t) - m * G * d * math.sin(t)  # noqa: E731
    lo, hi = 0.0, target
    for _ in range(100):  # bisection on the balance
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if f(mid) > 0.0 else (lo, mid)
    assert abs(art[pk.C["A_Q"]] - 0.5 * (lo + hi)) < 1e-5
    assert abs(art[pk.C["A_QD"]]) < 1e-4


def test_revolute_limit_holds(oracle_lib):
    pk = _pendulum(limits=(-0.3, 0.3))
    o = oracle_lib.OracleSim(pk)
    o.write("art", pk.C["A_QD"], [4.0])  # enough to swing past 1 rad without the limit
    q = []
    for _ in range(480):
        o.step(1)
        q.append(o.read("art")[pk.C["A_Q"]])
    q = np.array(q)
    assert q.max() <= 0.3 + 1e-4 and q.min() >= -0.3 - 1e-4
    assert q.max() > 0.29  # it did reach the limit


def test_prismatic_slide_follows_the_euler_recurrence(oracle_lib):
    axis = np.array([1.0, 0.0, -1.0]) / math.sqrt(2.0)
    b = SceneBuilder(fps=240)
    body = b.add_body(xform=[0.0, 0.0, 2.0, 0, 0, 0, 1])
    b.add_shape_sphere(body, radius=0.05)
    b.add_joint_prismatic(-1, body, axis=list(axis), parent_xform=[0.0, 0.0, 2.0, 0, 0, 0, 1])
    pk = pack(b.finalize())
    o = oracle_lib.OracleSim(pk)
    o.step(120)
    dt = np.float32(1.0 / (240 * pk.params["substeps"]))
    a = np.float32(G * -axis[2])
    v = x = np.float32(0.0)
    for _ in range(120 * pk.params["substeps"]):
        v = np.float32(v + a * dt)
        x = np.float32(x + v * dt)
    art = o.read("art")
    assert art[pk.C["A_Q"]] == x and art[pk.C["A_QD"]] == v


def test_conical_pendulum_on_a_ball_joint(oracle_lib):
    L, th = 0.6, 0.5
    omega = math.sqrt(G / (L * math.cos(th)))
    b = SceneBuilder(fps=240)
    bob = b.add_body(xform=[0.0, 0.0, 2.0 - L, 0, 0, 0, 1])
    b.add_shape_sphere(bob, radius=0.02)
    b.add_joint_ball(-1, bob, parent_xform=[0.0, 0.0, 2.0, 0, 0, 0, 1], child_xform=[0.0, 0.0, L, 0, 0, 0, 1],
                     q=[0.0, math.sin(th / 2), 0.0, math.cos(th / 2)])
    pk = pack(b.finalize())
    o = oracle_lib.OracleSim(pk)
    o.write("art", pk.C["A_QD"], [0.0, 0.0, omega])  # a ball joint's speed is its angular velocity (world)
    period = 2.0 * math.pi / omega
    frames = int(2.0 * period * 240)
    cone, azimuth = [], []
    for _ in range(frames):
        o.step(1)
        p = o.body_poses()[0, :3].astype(np.float64) - np.array([0.0, 0.0, 2.0])
        cone.append(math.acos(-p[2] / np.linalg.norm(p)))
        azimuth.append(math.atan2(p[1], p[0]))
    cone = np.array(cone)
    assert np.abs(cone - th).max() < 1e-4
    rate = (np.unwrap(azimuth)[-1] - np.unwrap(azimuth)[0]) / ((frames - 1) / 240.0)
    assert abs(rate - omega) / omega < 1e-3


def test_pd_arm_static_equilibrium(oracle_lib):
    ell, ke, kd = 0.3, 300.0, 20.0
    targets, masses = [0.6, -0.4, 0.8], [1.0, 0.7, 0.4]
    b = SceneBuilder(fps=240)
    parent = -1
    for k in range(3):
        body = b.add_body(xform=[0.0, 0.0, 2.0 - ell * (k + 0.5), 0, 0, 0, 1])
        b.add_shape_capsule(body, radius=0.02, half_height=0.1, mass=masses[k])
        b.add_joint_revolute(parent, body, axis=[0, 1, 0],
                             parent_xform=[0.0, 0.0, -ell / 2 if parent >= 0 else 2.0, 0, 0, 0, 1],
                             child_xform=[0.0, 0.0, ell / 2, 0, 0, 0, 1], targetKe=ke, targetKd=kd,
                             targetPos=targets[k])
        parent = body
    pk = pack(b.finalize())
    C = pk.C
    o = oracle_lib.OracleSim(pk)
    o.step(2400)
    art = o.read("art").astype(np.float64)
    q, qd = art[C["A_Q"]:C["A_Q"] + 3], art[C["A_QD"]:C["A_QD"] + 3]
    poses = o.body_poses().astype(np.float64)
    rec = pk.statF.reshape(-1, 4)[C["SF_BODY"]:C["SF_BODY"] + pk.NB * 8].astype(np.float64).reshape(pk.NB, 8, 4)
    mass = 1.0 / rec[:, 0, 0]
    joint_x = [poses[k, 0] + (_qmat(poses[k, 4:8]) @ np.array([0.0, 0.0, ell / 2]))[0] for k in range(3)]
    for i in range(3):
        gravity = sum(mass[j] * G * (poses[j, 0] - joint_x[i]) for j in range(i, 3))  # torque about +y
        assert abs(gravity) > 0.3
        assert abs(ke * (targets[i] - q[i]) - kd * qd[i] + gravity) < 1e-5
