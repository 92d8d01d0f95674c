"""Small seeded scenes covering the features of the hot path, built with the SceneBuilder mirror."""
import math

import numpy as np

from steel_webgpu_b200 import SceneBuilder, synth


def boxes(n=64, seed=1):
    return synth.boxes_on_plane(n, seed=seed)


def mixed_prims(seed=3, n=24):
    """Boxes, spheres, capsules, cylinders and random hulls (<= 16 and > 16 points) on a plane."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240)
    b.add_ground_plane(mu=0.7)
    for i in range(n):
        p = [float(rng.uniform(-0.6, 0.6)), float(rng.uniform(-0.6, 0.6)), 0.15 + 0.22 * i]
        body = b.add_body(xform=p + synth._rand_quat(rng))
        k = i % 6
        if k == 0:
            b.add_shape_box(body, hx=0.08, hy=0.05, hz=0.06, mu=0.6)
        elif k == 1:
            b.add_shape_sphere(body, radius=0.06, mu=0.5)
        elif k == 2:
            b.add_shape_capsule(body, radius=0.04, half_height=0.07, mu=0.6)
        elif k == 3:
            b.add_shape_cylinder(body, radius=0.05, half_height=0.06, mu=0.6)
        elif k == 4:
            b.add_shape_convex_hull(body, vertices=synth._ellipsoid_points(rng, 12), mu=0.6)
        else:
            b.add_shape_convex_hull(body, vertices=synth._ellipsoid_points(rng, 24), mu=0.6)
    return b.finalize()


def articulated(seed=5):
    """Two quadrupeds with PD drives and limits, one hanging revolute chain, a D6 and a ball pendulum."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=500)
    b.add_ground_plane(mu=0.8)
    synth._add_quadruped(b, rng, [0.0, 0.0, 0.9])
    synth._add_quadruped(b, rng, [1.5, 0.0, 0.9])
    synth._add_chain(b, rng, [3.0, 0.0, 2.2], 8, ratio_max=100.0)
    base = b.add_body(xform=[-1.5, 0, 1.0, 0, 0, 0, 1])
    b.add_shape_box(base, hx=0.1, hy=0.1, hz=0.1)
    b.add_joint_fixed(-1, base, parent_xform=[-1.5, 0, 1.0, 0, 0, 0, 1])
    arm = b.add_body(xform=[-1.5, 0, 0.7, 0, 0, 0, 1])
    b.add_shape_capsule(arm, radius=0.03, half_height=0.12)
    b.add_joint_d6(base, arm, linear_axes=[[0, 0, 1]], angular_axes=[[1, 0, 0], [0, 1, 0]],
                   parent_xform=[0, 0, -0.1, 0, 0, 0, 1], child_xform=[0, 0, 0.2, 0, 0, 0, 1], q=[0.0, 0.3, -0.2])
    bob = b.add_body(xform=[-2.5, 0, 1.5, 0, 0, 0, 1])
    b.add_shape_sphere(bob, radius=0.08)
    b.add_joint_ball(-1, bob, parent_xform=[-2.5, 0, 2.0, 0, 0, 0, 1], child_xform=[0, 0, 0.4, 0, 0, 0, 1],
                     q=[math.sin(0.2), 0.0, 0.0, math.cos(0.2)])
    return b.finalize()


def chains_and_quads(seed=7, n_quad=4, chain_links=40):
    """Quadrupeds plus one 40-link chain with link mass ratios up to 1e3 (the articulation workload)."""
    return synth.quadrupeds(n_quad=n_quad, n_chains=1, chain_links=chain_links, seed=seed)


def hull_bin(seed=11, n=160):
    """Hulls, boxes and capsules poured into a bin of 5 static boxes (the convex-pour workload)."""
    return synth.convex_pour(n=n, seed=seed, bin_size=1.5, layer=0.25)


def small_batch(seed=13, n=6):
    """Independent scenes of uneven size (the uneven-batch workload)."""
    return synth.uneven_batch(n_scenes=n, seed=seed, lo=8, hi=96, chain_lo=2, chain_hi=12)


def vel_limited(seed=17):
    """A 10-link revolute chain released from a steep angle with joint velocity limits of 2 rad/s
    (enable_joint_velocity_limits), next to a PD-driven quadruped without limits."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240)
    b.add_ground_plane(mu=0.7)
    parent = -1
    top = [0.0, 0.0, 2.5]
    for k in range(10):
        body = b.add_body(xform=[top[0], top[1], top[2] - 0.1 * (k + 0.5), 0, 0, 0, 1])
        b.add_shape_capsule(body, radius=0.02, half_height=0.04, mass=float(0.1 * math.exp(rng.uniform(0.0, 2.0))))
        b.add_joint_revolute(parent, body, axis=[0, 1, 0],
                             parent_xform=[0, 0, -0.05, 0, 0, 0, 1] if parent >= 0 else top + [0, 0, 0, 1],
                             child_xform=[0, 0, 0.05, 0, 0, 0, 1], q=[1.3] if k == 0 else [0.2], velocityLimit=2.0)
        parent = body
    synth._add_quadruped(b, rng, [1.5, 0.0, 0.9])
    return b.finalize(solver=dict(enable_joint_velocity_limits=True))


def sleepers(seed=19):
    """Sleeping on (enable_sleeping): boxes resting on the plane and a two-box stack settle and fall
    asleep, a 4-link revolute chain hangs at rest from the world (a fixed-base island), and a box
    dropped from 2.4 m lands on the stack after about 0.7 s and wakes its island."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.6)
    for i in range(3):
        body = b.add_body(xform=[-1.0 + 0.5 * i, 0.8, 0.101, 0, 0, 0, 1])
        h = float(rng.uniform(0.08, 0.12))
        b.add_shape_box(body, hx=h, hy=h, hz=0.1, mu=0.6)
    lo = b.add_body(xform=[0.0, 0.0, 0.1, 0, 0, 0, 1])
    b.add_shape_box(lo, hx=0.2, hy=0.2, hz=0.1, mu=0.6)
    hi = b.add_body(xform=[0.0, 0.0, 0.3, 0, 0, 0, 1])
    b.add_shape_box(hi, hx=0.15, hy=0.15, hz=0.1, mu=0.6)
    drop = b.add_body(xform=[0.02, 0.01, 2.8, 0, 0, 0, 1])
    b.add_shape_box(drop, hx=0.08, hy=0.08, hz=0.08, mu=0.6)
    parent = -1
    top = [1.2, -0.8, 1.5]
    for k in range(4):
        body = b.add_body(xform=[top[0], top[1], top[2] - 0.1 * (k + 0.5), 0, 0, 0, 1])
        b.add_shape_capsule(body, radius=0.02, half_height=0.04, mass=0.2)
        b.add_joint_revolute(parent, body, axis=[0, 1, 0],
                             parent_xform=[0, 0, -0.05, 0, 0, 0, 1] if parent >= 0 else top + [0, 0, 0, 1],
                             child_xform=[0, 0, 0.05, 0, 0, 0, 1])
        parent = body
    return b.finalize(solver=dict(enable_sleeping=True))


def momentum_stack(seed=23):
    """nesterov_momentum on: a five-box stack whose masses grow 10^0.75 per box (a 10^3 ratio,
    heavy on light) and a PD-held quadruped standing on the plane (contact impulses on links);
    friction joins at iteration 8 (contact_friction_position_iterations=4), so the restart at
    that iteration runs too."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.7)
    for k in range(5):
        body = b.add_body(xform=[0.0, 0.0, 0.1 + 0.2 * k + 0.002 * k, 0, 0, 0, 1])
        b.add_shape_box(body, hx=0.15, hy=0.15, hz=0.1, mu=0.7, mass=float(0.2 * 10.0 ** (0.75 * k)))
    synth._add_quadruped(b, rng, [1.2, 0.0, 0.9])
    return b.finalize(solver=dict(nesterov_momentum=True, contact_friction_position_iterations=4))


def spinners(seed=29):
    """Contact torsion: articulated plates spinning flat on the plane whose shapes have a torsion
    radius (min_torsional_patch_radius), so each plate's coplanar contact cluster gets a spin row
    that shares the Coulomb budget with sliding: a plate with a hinged tab, a sliding plate with a
    hinged flap, and a free-body plate (no spin row: torsion rows are articulated-only)."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.8)
    spun = []
    p0 = b.add_body(xform=[0.0, 0.0, 0.05, 0, 0, 0, 1], twist=[0.0, 0.0, 0.0, 0.0, 0.0, 6.0])
    spun.append(b.add_shape_box(p0, hx=0.2, hy=0.15, hz=0.05, mu=0.8))
    b.add_joint_free(p0)
    tab = b.add_body(xform=[0.0, 0.2, 0.05, 0, 0, 0, 1])
    b.add_shape_box(tab, hx=0.05, hy=0.05, hz=0.02, mu=0.8)
    b.add_joint_revolute(p0, tab, axis=[1, 0, 0], parent_xform=[0.0, 0.15, 0.0, 0, 0, 0, 1],
                         child_xform=[0.0, -0.05, 0.0, 0, 0, 0, 1])
    p1 = b.add_body(xform=[1.0, 0.0, 0.04, 0, 0, 0, 1], twist=[0.3, 0.0, 0.0, 0.0, 0.0, -4.0])
    spun.append(b.add_shape_box(p1, hx=0.15, hy=0.15, hz=0.04, mu=0.8))
    b.add_joint_free(p1)
    flap = b.add_body(xform=[1.25, 0.0, 0.02, 0, 0, 0, 1])
    spun.append(b.add_shape_box(flap, hx=0.1, hy=0.12, hz=0.02, mu=0.8))
    b.add_joint_revolute(p1, flap, axis=[0, 1, 0], parent_xform=[0.15, 0.0, -0.02, 0, 0, 0, 1],
                         child_xform=[-0.1, 0.0, 0.0, 0, 0, 0, 1])
    f = b.add_body(xform=[-1.0, 0.0, 0.05, 0, 0, 0, 1], twist=[0.0, 0.0, 0.0, 0.0, 0.0, 5.0])
    spun.append(b.add_shape_box(f, hx=0.2, hy=0.15, hz=0.05, mu=0.8))
    sc = b.finalize()
    for s in sc.json["shapes"]:
        if s["sid"] in spun:
            s["torsion_radius"] = float(rng.uniform(0.08, 0.12))
    return sc


def compliant(seed=31):
    """contact_compliance on: boxes of three stiffnesses (ke 1e3, 1e4, 1e5 with damping kd) dropped
    on a stiff plane; their normal rows are spring-dampers, and the body-pair reduction keeps every
    point."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.6, ke=1e7, kd=0.0)
    for i, (ke, kd) in enumerate(((1e3, 20.0), (1e4, 60.0), (1e5, 200.0), (1e4, 60.0))):
        body = b.add_body(xform=[-0.9 + 0.6 * i, 0.0, 0.3 + 0.2 * i] + synth._rand_quat(rng))
        b.add_shape_box(body, hx=0.1, hy=0.08, hz=0.06, mu=0.6, ke=ke, kd=kd)
    return b.finalize(solver=dict(contact_compliance=True, enable_restitution=False))


def velocity_pass(seed=37):
    """velocity_iterations=4: a stack of boxes that starts 3 mm interpenetrated (a depenetration the
    position sweeps push out, the velocity sweeps then clear of bias), friction anchors on, and a
    6-link revolute chain with +-0.4 rad joint limits released from 1 rad, whose links hit each
    other (dense rows) and their limits (limit rows) while the velocity pass runs without bias."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.7)
    for k in range(4):
        body = b.add_body(xform=[0.01 * float(rng.uniform(-1, 1)), 0.0, 0.097 + 0.197 * k, 0, 0, 0, 1])
        b.add_shape_box(body, hx=0.15, hy=0.12, hz=0.1, mu=0.7)
    parent = -1
    top = [1.0, 0.0, 1.2]
    for k in range(6):
        body = b.add_body(xform=[top[0], top[1], top[2] - 0.1 * (k + 0.5), 0, 0, 0, 1])
        b.add_shape_capsule(body, radius=0.03, half_height=0.04, mass=0.3)
        b.add_joint_revolute(parent, body, axis=[0, 1, 0],
                             parent_xform=[0, 0, -0.05, 0, 0, 0, 1] if parent >= 0 else top + [0, 0, 0, 1],
                             child_xform=[0, 0, 0.05, 0, 0, 0, 1], q=[1.0] if k == 0 else [0.3],
                             limitLower=-0.4 if k else -2.0, limitUpper=0.4 if k else 2.0)
        parent = body
    return b.finalize(solver=dict(velocity_iterations=4))


def load_friction(seed=41):
    """Joint friction with a load coefficient (enable_joint_friction, friction_load_coefficient): two
    pendulums released from 1.2 rad, one whose friction bound grows with the force its joint
    transmits (0.3 per newton) and holds it, one with plain friction that swings."""
    b = SceneBuilder(fps=240)
    for i in range(2):
        top = [0.8 * i, 0.0, 1.5]
        body = b.add_body(xform=[top[0], 0.0, top[2] - 0.3, 0, 0, 0, 1])
        b.add_shape_box(body, hx=0.04, hy=0.04, hz=0.25, mass=1.0)
        b.add_joint_revolute(-1, body, axis=[0, 1, 0], parent_xform=top + [0, 0, 0, 1],
                             child_xform=[0, 0, 0.3, 0, 0, 0, 1], q=[1.2], friction=0.2)
    sc = b.finalize(solver=dict(enable_joint_friction=True))
    sc.json["joints"]["friction_load_coefficient"] = [0.3, 0.0]
    return sc


def spin_roll(seed=43):
    """Torsional and rolling friction of free bodies (free_rigid_torsional_friction 0.05,
    free_rigid_rolling_friction 0.01): a box spinning flat on the plane and spheres rolling on it
    come to rest through the spin row and the rolling pair of each contact."""
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.6)
    box = b.add_body(xform=[0.0, 0.0, 0.05, 0, 0, 0, 1], twist=[0.0, 0.0, 0.0, 0.0, 0.0, 8.0])
    b.add_shape_box(box, hx=0.15, hy=0.1, hz=0.05, mu=0.6)
    for i, v in enumerate((1.0, 2.0)):
        r = 0.08
        ball = b.add_body(xform=[-0.6, 0.4 * i - 0.2, r, 0, 0, 0, 1], twist=[v, 0.0, 0.0, 0.0, v / r, 0.0])
        b.add_shape_sphere(ball, radius=r, mu=0.6)
    return b.finalize(solver=dict(free_rigid_torsional_friction=0.05, free_rigid_rolling_friction=0.01))


def ang_art(seed=47, cone="elliptic", creep=0.0, relaxation=1.0):
    """Torsional and rolling friction of articulated contacts (enable_torsional_rolling_friction,
    friction_anchor_beta 0): two free-floating dumbbells (two spheres on a fixed joint), one spinning
    flat about the vertical and one rolling across its bar, and a quadruped dropped on its feet. Every contact that
    touches a link runs the 5-row angular block (t1, t2, spin, roll1, roll2) on the chosen cone."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240)
    mat = dict(muTorsional=0.05, muRolling=0.02)
    b.add_ground_plane(mu=0.7, **mat)
    r = 0.08
    for i, tw in enumerate(([0.0, 0.0, 0.0, 0.0, 0.0, 6.0], [0.0, 1.0, 0.0, -1.0 / r, 0.0, 0.0])):
        y = 0.6 * i
        left = b.add_body(xform=[-0.15, y, r, 0, 0, 0, 1], twist=tw)
        b.add_shape_sphere(left, radius=r, mu=0.6, **mat)
        b.add_joint_free(left)
        right = b.add_body(xform=[0.15, y, r, 0, 0, 0, 1])
        b.add_shape_sphere(right, radius=r, mu=0.6, **mat)
        b.add_shape_capsule(right, radius=0.02, half_height=0.1, mu=0.6,
                            xform=[-0.15, 0, 0, 0, math.sin(math.pi / 4), 0, math.cos(math.pi / 4)], **mat)
        b.add_joint_fixed(left, right, parent_xform=[0.3, 0, 0, 0, 0, 0, 1])
    synth._add_quadruped(b, rng, [0.0, 1.6, 0.9])
    return b.finalize(solver=dict(enable_torsional_rolling_friction=True, friction_anchor_beta=0.0,
                                  torsional_rolling_friction_cone=cone,
                                  torsional_rolling_friction_creep_speed=creep, relaxation=relaxation))


def four_bar(seed=53):
    """A parallelogram four-bar linkage (crank, coupler and rocker on revolute joints, closed by a
    loop joint from the world to the rocker), released at 0.5 rad so that the pendulum hung from its coupler swings into the ground, beside a
    quadruped with PD drives and limits: loop-closure dense rows, joint rows and contacts in one scene."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240)
    b.add_ground_plane(mu=0.8)
    y = [0, 1, 0]
    crank = b.add_body(xform=[0.0, 0.0, 0.32, 0, 0, 0, 1])
    b.add_shape_box(crank, hx=0.02, hy=0.02, hz=0.1, mass=0.5)
    b.add_joint_revolute(-1, crank, axis=y, parent_xform=[0.0, 0.0, 0.42, 0, 0, 0, 1],
                         child_xform=[0, 0, 0.1, 0, 0, 0, 1], q=[0.5])
    coupler = b.add_body(xform=[0.3, 0.0, 0.22, 0, 0, 0, 1])
    b.add_shape_box(coupler, hx=0.3, hy=0.02, hz=0.02, mass=0.5)
    b.add_joint_revolute(crank, coupler, axis=y, parent_xform=[0, 0, -0.1, 0, 0, 0, 1],
                         child_xform=[-0.3, 0, 0, 0, 0, 0, 1], q=[-0.5])
    rocker = b.add_body(xform=[0.6, 0.0, 0.32, 0, 0, 0, 1])
    b.add_shape_box(rocker, hx=0.02, hy=0.02, hz=0.1, mass=0.5)
    b.add_joint_revolute(coupler, rocker, axis=y, parent_xform=[0.3, 0, 0, 0, 0, 0, 1],
                         child_xform=[0, 0, -0.1, 0, 0, 0, 1], q=[0.5])
    b.add_joint_revolute(-1, rocker, axis=y, parent_xform=[0.6, 0.0, 0.42, 0, 0, 0, 1],
                         child_xform=[0, 0, 0.1, 0, 0, 0, 1])
    tip = b.add_body(xform=[0.3, 0.0, 0.07, 0, 0, 0, 1])
    b.add_shape_sphere(tip, radius=0.05, mass=2.0)
    b.add_joint_revolute(coupler, tip, axis=[1, 0, 0], parent_xform=[0, 0, -0.05, 0, 0, 0, 1],
                         child_xform=[0, 0, 0.15, 0, 0, 0, 1], q=[0.4])
    synth._add_quadruped(b, rng, [1.5, 0.0, 0.9])
    return b.finalize()


def mimic_arms(seed=59):
    """Mimic joints (set_joint_mimic): a fixed base with a PD-driven arm and a second arm that
    follows it at q2 = 0.1 - q1, and a two-finger gripper whose second finger mirrors the first on
    prismatic joints; the arms sweep through boxes resting on the ground."""
    b = SceneBuilder(fps=240)
    b.add_ground_plane(mu=0.8)
    base = b.add_body(xform=[0.0, 0.0, 0.45, 0, 0, 0, 1])
    b.add_shape_box(base, hx=0.05, hy=0.05, hz=0.05, mass=2.0)
    b.add_joint_fixed(-1, base, parent_xform=[0.0, 0.0, 0.45, 0, 0, 0, 1])
    arms = []
    for side in (-1, 1):
        arm = b.add_body(xform=[0.0, 0.12 * side, 0.25, 0, 0, 0, 1])
        b.add_shape_capsule(arm, radius=0.03, half_height=0.17, mass=0.6)
        arms.append(b.add_joint_revolute(base, arm, axis=[0, 1, 0], parent_xform=[0, 0.12 * side, 0, 0, 0, 0, 1],
                                         child_xform=[0, 0, 0.2, 0, 0, 0, 1], targetKe=40.0, targetKd=2.0,
                                         targetPos=0.9 if side < 0 else 0.0, limitLower=-1.5, limitUpper=1.5))
    b.set_joint_mimic(arms[1], arms[0], coeffs=(0.1, -1.0))
    fingers = []
    for side in (-1, 1):
        f = b.add_body(xform=[0.0, 0.04 * side, 0.36, 0, 0, 0, 1])
        b.add_shape_box(f, hx=0.01, hy=0.01, hz=0.03, mass=0.1)
        fingers.append(b.add_joint_prismatic(base, f, axis=[0, 1, 0], parent_xform=[0, 0.04 * side, -0.09, 0, 0, 0, 1],
                                             targetKe=20.0, targetKd=1.0, targetPos=-0.02 * side, limitLower=-0.03,
                                             limitUpper=0.03))
    b.set_joint_mimic(fingers[1], fingers[0], coeffs=(0.0, -1.0))
    rng = np.random.default_rng(seed)
    for i in range(6):
        bx = b.add_body(xform=[float(rng.uniform(-0.35, 0.35)), float(rng.uniform(-0.2, 0.2)), 0.05 + 0.11 * (i % 2),
                               0, 0, 0, 1])
        b.add_shape_box(bx, hx=0.05, hy=0.05, hz=0.05, mass=0.3)
    return b.finalize()


def controlled(seed=61):
    """The user-control surface: two PD-driven quadrupeds and a hanging revolute chain (joint
    targets and forces), plus free boxes on the plane and one in the air (body wrench, pose and
    twist)."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.7)
    synth._add_quadruped(b, rng, [0.0, 0.0, 0.9])
    synth._add_quadruped(b, rng, [1.5, 0.0, 0.9])
    synth._add_chain(b, rng, [3.0, 0.0, 2.2], 6, ratio_max=10.0)
    for i in range(3):
        body = b.add_body(xform=[-1.0 - 0.5 * i, 0.5, 0.101, 0, 0, 0, 1])
        b.add_shape_box(body, hx=0.1, hy=0.1, hz=0.1, mu=0.6)
    body = b.add_body(xform=[-2.0, -1.0, 1.5, 0, 0, 0, 1])
    b.add_shape_box(body, hx=0.08, hy=0.12, hz=0.1, mu=0.6)
    return b.finalize()


def box_carpet(n=2200, seed=67, spacing=0.35):
    """n small boxes in a grid, each resting 1 mm into the plane and too far apart to touch: four
    plane contacts per box, so the contact count passes the block sort's 8192 shared-memory keys
    and the radix sort runs."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.6)
    side = int(math.ceil(math.sqrt(n)))
    for i in range(n):
        x, y = (i % side - side / 2) * spacing, (i // side - side / 2) * spacing
        h = float(rng.uniform(0.03, 0.05))
        body = b.add_body(xform=[x, y, h - 0.001, 0, 0, 0, 1])
        b.add_shape_box(body, hx=h, hy=h, hz=h, mu=0.6)
    return b.finalize()
