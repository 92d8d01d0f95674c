"""Seeded synthetic scenes with the shapes of the benchmark workloads.

No public dataset exists for this path; these generators build scenes through the
``SceneBuilder`` mirror with the sizes and distributions of the workloads:

* ``boxes_on_plane``   64 boxes, half-extents U[0.05, 0.15] m, density 1000, positions in a
                       2x2x2 m volume above a ground plane, random orientations, mu 0.6, e 0,
                       240 fps, 4 substeps, 12 iterations.
* ``convex_pour``      8192 convex bodies (50 % hulls of 8-32 points on ellipsoids with semi-axes
                       U[0.03, 0.1], 25 % boxes, 25 % capsules r U[0.02, 0.05], half-length
                       U[0.02, 0.08]) poured into a 4x4 m bin of 5 static boxes, 240 fps.
* ``quadrupeds``       quadruped-like floating-base articulations (0.5x0.3x0.1 m 10 kg base, 4
                       legs of 3 revolute joints, capsule links r 0.03, length U[0.2, 0.25], mass
                       U[0.5, 1.5]) with PD targets, plus 40-link revolute chains with link mass
                       ratios log-U[1, 1e3], on a ground plane, 500 fps.
* ``uneven_batch``     a list of independent scenes with log-U[8, 512] bodies from the box mix,
                       each with one revolute chain of U[2, 40] links and its own ground plane.

Every draw comes from one ``numpy.random.default_rng(seed)``. Box hulls are built directly
(``builder.box_hull``) rather than by quickhull, for generation speed at batch scale.
"""
from __future__ import annotations

import math

import numpy as np

from .builder import SceneBuilder


def _rand_quat(rng):
    """Uniform random unit quaternion (x, y, z, w), Shoemake's method."""
    u1, u2, u3 = rng.random(3)
    a, b = math.sqrt(1 - u1), math.sqrt(u1)
    return [a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2),
            b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3)]


def boxes_on_plane(n=64, seed=0, fps=240, substeps=4, iterations=12, volume=2.0, z0=0.2, mu=0.6):
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=fps, box_hulls="direct")
    b.add_ground_plane(mu=mu)
    placed = []
    for _ in range(n):
        he = rng.uniform(0.05, 0.15, 3)
        rad = float(np.linalg.norm(he))
        # Placements whose bounding spheres overlap an earlier box are redrawn (no start in contact).
        for _try in range(1000):
            p = [rng.uniform(-volume / 2, volume / 2), rng.uniform(-volume / 2, volume / 2), z0 + rng.uniform(0, volume)]
            if all(math.dist(p, q) > rad + r for q, r in placed):
                break
        placed.append((p, rad))
        body = b.add_body(xform=p + _rand_quat(rng))
        b.add_shape_box(body, hx=float(he[0]), hy=float(he[1]), hz=float(he[2]), mu=mu, density=1000.0)
    return b.finalize(solver=dict(substeps=substeps, iterations=iterations))


def _ellipsoid_points(rng, k):
    axes = rng.uniform(0.03, 0.1, 3)
    v = rng.normal(size=(k, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * axes).tolist()


def convex_pour(n=8192, seed=0, fps=240, substeps=4, iterations=12, bin_size=4.0, wall_h=1.0, layer=0.25):
    """Bodies on a jittered lattice above a 4x4 m bin (floor + 4 walls, 5 static boxes)."""
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=fps, box_hulls="direct")
    half = bin_size / 2
    t = 0.1
    walls = [([0, 0, -t], [half + t, half + t, t]),
             ([half + t / 2, 0, wall_h / 2], [t / 2, half + t, wall_h / 2]),
             ([-half - t / 2, 0, wall_h / 2], [t / 2, half + t, wall_h / 2]),
             ([0, half + t / 2, wall_h / 2], [half, t / 2, wall_h / 2]),
             ([0, -half - t / 2, wall_h / 2], [half, t / 2, wall_h / 2])]
    for pos, he in walls:
        b.add_shape_box(-1, hx=he[0], hy=he[1], hz=he[2], xform=list(pos) + [0, 0, 0, 1], mu=0.6)
    per_row = int(bin_size / layer) - 1
    per_layer = per_row * per_row
    for i in range(n):
        lz, rem = divmod(i, per_layer)
        ix, iy = divmod(rem, per_row)
        p = [-half + layer * (ix + 1) + rng.uniform(-0.02, 0.02), -half + layer * (iy + 1) + rng.uniform(-0.02, 0.02),
             0.2 + layer * lz + rng.uniform(0, 0.05)]
        body = b.add_body(xform=p + _rand_quat(rng))
        kind = rng.random()
        if kind < 0.5:
            b.add_shape_convex_hull(body, vertices=_ellipsoid_points(rng, int(rng.integers(8, 33))), mu=0.6)
        elif kind < 0.75:
            he = rng.uniform(0.03, 0.1, 3)
            b.add_shape_box(body, hx=float(he[0]), hy=float(he[1]), hz=float(he[2]), mu=0.6)
        else:
            b.add_shape_capsule(body, radius=float(rng.uniform(0.02, 0.05)), half_height=float(rng.uniform(0.02, 0.08)),
                                mu=0.6)
    return b.finalize(solver=dict(substeps=substeps, iterations=iterations))


def _add_chain(b, rng, base_pos, n_links, link_len=0.1, radius=0.02, ratio_max=1e3, ke=0.0, kd=0.0):
    """A serial revolute chain hanging from the world; link masses log-U[1, ratio_max] x 0.1 kg."""
    parent = -1
    x = list(base_pos)
    for k in range(n_links):
        m = 0.1 * math.exp(rng.uniform(0.0, math.log(ratio_max)))
        body = b.add_body(xform=[x[0], x[1], x[2] - link_len * (k + 0.5), 0, 0, 0, 1])
        b.add_shape_capsule(body, radius=radius, half_height=link_len * 0.4, mass=m)
        b.add_joint_revolute(parent, body, axis=[0, 1, 0] if k % 2 == 0 else [1, 0, 0],
                             parent_xform=[0, 0, -link_len * 0.5, 0, 0, 0, 1] if parent >= 0
                             else [x[0], x[1], x[2], 0, 0, 0, 1],
                             child_xform=[0, 0, link_len * 0.5, 0, 0, 0, 1], targetKe=ke, targetKd=kd)
        parent = body
    return parent


def _add_quadruped(b, rng, pos, ke=60.0, kd=2.0):
    base = b.add_body(xform=list(pos) + [0, 0, 0, 1])
    b.add_shape_box(base, hx=0.25, hy=0.15, hz=0.05, mass=10.0)
    dofs = []
    for sx in (-1, 1):
        for sy in (-1, 1):
            parent = base
            px, py = 0.2 * sx, 0.13 * sy
            for seg in range(3):
                L = float(rng.uniform(0.2, 0.25))
                m = float(rng.uniform(0.5, 1.5))
                link = b.add_body(xform=[pos[0] + px, pos[1] + py, pos[2] - 0.05 - L * (seg + 0.5), 0, 0, 0, 1])
                b.add_shape_capsule(link, radius=0.03, half_height=max(L / 2 - 0.03, 0.01), mass=m)
                axis = [1, 0, 0] if seg == 0 else [0, 1, 0]
                pxf = [px, py, -0.05, 0, 0, 0, 1] if seg == 0 else [0, 0, -prevL / 2, 0, 0, 0, 1]
                j = b.add_joint_revolute(parent, link, axis=axis, parent_xform=pxf,
                                         child_xform=[0, 0, L / 2, 0, 0, 0, 1], targetKe=ke, targetKd=kd,
                                         limitLower=-1.5, limitUpper=1.5)
                dofs.append(j)
                parent = link
                prevL = L
    return dofs


def quadrupeds(n_quad=1024, n_chains=64, chain_links=40, seed=0, fps=500, substeps=4, iterations=12, spacing=1.2):
    rng = np.random.default_rng(seed)
    b = SceneBuilder(fps=fps, box_hulls="direct")
    b.add_ground_plane(mu=0.8)
    side = int(math.ceil(math.sqrt(n_quad + n_chains)))
    joints = []
    k = 0
    for i in range(n_quad):
        gx, gy = divmod(k, side)
        k += 1
        joints.extend(_add_quadruped(b, rng, [gx * spacing, gy * spacing, 0.85]))
    for i in range(n_chains):
        gx, gy = divmod(k, side)
        k += 1
        _add_chain(b, rng, [gx * spacing, gy * spacing, chain_links * 0.1 + 0.5], chain_links)
    scene = b.finalize(solver=dict(substeps=substeps, iterations=iterations))
    scene.json["info"] = dict(pd_joints=[b.joint_dof(j) for j in joints])
    return scene


def uneven_batch(n_scenes=2048, seed=0, fps=240, substeps=4, iterations=12, lo=8, hi=512, chain_lo=2, chain_hi=40):
    rng = np.random.default_rng(seed)
    scenes = []
    for s in range(n_scenes):
        nb = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        b = SceneBuilder(fps=fps, box_hulls="direct")
        b.add_ground_plane(mu=0.6)
        side = max(int(math.ceil(math.sqrt(nb))), 1)
        for i in range(nb):
            gx, gy = divmod(i, side)
            he = rng.uniform(0.05, 0.15, 3)
            p = [gx * 0.4 - side * 0.2, gy * 0.4 - side * 0.2, 0.3 + rng.uniform(0, 1.0)]
            body = b.add_body(xform=p + _rand_quat(rng))
            b.add_shape_box(body, hx=float(he[0]), hy=float(he[1]), hz=float(he[2]), mu=0.6)
        _add_chain(b, rng, [side * 0.2 + 1.0, 0.0, 4.5], int(rng.integers(chain_lo, chain_hi + 1)), ratio_max=10.0)
        scenes.append(b.finalize(solver=dict(substeps=substeps, iterations=iterations)))
    return scenes
