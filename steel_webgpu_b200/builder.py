"""Scene construction: a Python mirror of the reference's ``SceneBuilder``.

Follows ``packages/steel-webgpu/src/builder.js`` (Newton-style ModelBuilder):
``convexHull`` (quickhull, builder.js:61-173), analytic hull sample points
(builder.js:176-196), solid mass properties (builder.js:199-238) and
``finalize`` (builder.js:320-491), which returns the same ``LoadedScene``
shape that ``loadScene`` reads from ``scene.json`` + ``scene.bin``.

All arithmetic is IEEE double, as in JavaScript; arrays that the reference
stores in ``scene.bin`` are float32 / uint32 there and here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

JT = {"PRISMATIC": 0, "REVOLUTE": 1, "BALL": 2, "FIXED": 3, "FREE": 4, "DISTANCE": 5, "D6": 6}
GT = {"NONE": 0, "PLANE": 1, "HFIELD": 2, "SPHERE": 3, "CAPSULE": 4, "ELLIPSOID": 5, "CYLINDER": 6,
      "BOX": 7, "MESH": 8, "CONE": 9, "CONVEX_MESH": 10, "GAUSSIAN": 11}
UNLIMITED = 1e10
IDENTITY = [0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0]

# Newton's ShapeConfig defaults (builder.js:19-20); gap is ModelBuilder.rigid_gap.
SHAPE_DEFAULTS = dict(density=1000.0, mu=1.0, restitution=0.0, muTorsional=0.005, muRolling=0.0001, gap=0.1,
                      ke=2.5e3, kd=100.0, collisionGroup=1, world=-1, color=[0.7, 0.7, 0.7])
# Newton's JointDofConfig defaults (builder.js:22-23).
DOF_DEFAULTS = dict(limitLower=-UNLIMITED, limitUpper=UNLIMITED, targetPos=0.0, targetVel=0.0, targetKe=0.0,
                    targetKd=0.0, damping=0.0, armature=0.0, effortLimit=1e6, velocityLimit=1e6, friction=0.0)


# --- small rigid-transform math (double precision) -----------------------------------------
def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _add(a, b):
    return [a[0] + b[0], a[1] + b[1], a[2] + b[2]]


def _scale(a, s):
    return [a[0] * s, a[1] * s, a[2] * s]


def _norm(a):
    return math.hypot(a[0], a[1], a[2])


def qmul(a, b):
    return [a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1],
            a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0],
            a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3],
            a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2]]


def qconj(q):
    return [-q[0], -q[1], -q[2], q[3]]


def qrot(q, v):
    u = [q[0], q[1], q[2]]
    t = _scale(_cross(u, v), 2.0)
    return _add(_add(v, _scale(t, q[3])), _cross(u, t))


def qaxis(axis, angle):
    n = _norm(axis)
    s = math.sin(angle / 2.0) / n
    return [axis[0] * s, axis[1] * s, axis[2] * s, math.cos(angle / 2.0)]


def tmul(a, b):
    return _add(a[:3], qrot(a[3:], b[:3])) + qmul(a[3:], b[3:])


def tinv(t):
    qi = qconj(t[3:])
    return _scale(qrot(qi, t[:3]), -1.0) + qi


def qmat(q):
    x, y, z, w = q
    return [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
            2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
            2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]


def _js_round(x: float) -> float:
    """JavaScript Math.round: half-way cases go toward +infinity."""
    return math.floor(x + 0.5)


# --- convex hulls ---------------------------------------------------------------------------
def convex_hull(points):
    """Quickhull of a point cloud (builder.js:61-173).

    Returns ``{"verts": [[x,y,z]...], "faces": [{"n": [..], "d": d, "v": [...]}, ...]}`` with
    coplanar triangles merged into polygons, vertices counter-clockwise about the outward normal
    and each face plane ``n . x = d``.
    """
    seen = {}
    for p in points:
        k = (p[0], p[1], p[2])
        if k not in seen:
            seen[k] = [float(p[0]), float(p[1]), float(p[2])]
    P = list(seen.values())
    if len(P) < 4:
        raise ValueError("a convex hull needs at least 4 distinct points")
    lo = [math.inf] * 3
    hi = [-math.inf] * 3
    for p in P:
        lo = [min(lo[k], p[k]) for k in range(3)]
        hi = [max(hi[k], p[k]) for k in range(3)]
    eps = 1e-7 * max(_norm(_sub(hi, lo)), 1e-12)
    i0 = 0
    for i in range(1, len(P)):
        if P[i][0] < P[i0][0]:
            i0 = i

    def far(f):
        best, bd = -1, -1.0
        for i, p in enumerate(P):
            d = f(p)
            if d > bd:
                bd, best = d, i
        return best, bd

    i1, _ = far(lambda p: _norm(_sub(p, P[i0])))
    e = _sub(P[i1], P[i0])
    i2, d2 = far(lambda p: _norm(_cross(e, _sub(p, P[i0]))) / _norm(e))
    if d2 <= eps:
        raise ValueError("convex hull points are collinear")
    n0 = _cross(e, _sub(P[i2], P[i0]))
    i3, d3 = far(lambda p: abs(_dot(n0, _sub(p, P[i0]))) / _norm(n0))
    if d3 <= eps:
        raise ValueError("convex hull points are coplanar")
    center = _scale(_add(_add(P[i0], P[i1]), _add(P[i2], P[i3])), 0.25)

    class Face:
        __slots__ = ("v", "n", "d", "alive", "out", "vis", "group")

    def face(a, b, c):
        n = _cross(_sub(P[b], P[a]), _sub(P[c], P[a]))
        n = _scale(n, 1.0 / _norm(n))
        f = Face()
        f.v, f.n, f.d = [a, b, c], n, _dot(n, P[a])
        f.alive, f.out, f.vis, f.group = False, [], False, None
        return f

    def oriented(a, b, c):
        f = face(a, b, c)
        return face(a, c, b) if _dot(f.n, center) - f.d > 0 else f

    K = 1048576
    edges = {}

    def make(a, b, c):
        f = face(a, b, c)
        f.alive, f.out = True, []
        for k in range(3):
            edges[f.v[k] * K + f.v[(k + 1) % 3]] = f
        return f

    faces = [make(*oriented(i0, i1, i2).v), make(*oriented(i0, i1, i3).v),
             make(*oriented(i0, i2, i3).v), make(*oriented(i1, i2, i3).v)]

    def assign(pts, cands):
        for i in pts:
            best, bd = None, eps
            for f in cands:
                d = _dot(f.n, P[i]) - f.d
                if d > bd:
                    bd, best = d, f
            if best is not None:
                best.out.append(i)

    assign([i for i in range(len(P)) if i not in (i0, i1, i2, i3)], faces)
    for _guard in range(4 * len(P) + 16):
        f0 = next((f for f in faces if f.alive and f.out), None)
        if f0 is None:
            break
        p, pd = f0.out[0], -math.inf
        for i in f0.out:
            d = _dot(f0.n, P[i]) - f0.d
            if d > pd:
                pd, p = d, i
        f0.vis = True
        visible = [f0]
        seen_f = {id(f0)}
        horizon = []
        k = 0
        while k < len(visible):
            f = visible[k]
            k += 1
            for e_ in range(3):
                a, b = f.v[e_], f.v[(e_ + 1) % 3]
                nb = edges.get(b * K + a)
                if nb is None or id(nb) in seen_f:
                    if nb is not None and not nb.vis:
                        horizon.append((a, b))
                    continue
                if _dot(nb.n, P[p]) - nb.d > eps:
                    nb.vis = True
                    seen_f.add(id(nb))
                    visible.append(nb)
                else:
                    horizon.append((a, b))
        orphans = []
        for f in visible:
            f.alive = False
            for kk in range(3):
                key = f.v[kk] * K + f.v[(kk + 1) % 3]
                if edges.get(key) is f:
                    del edges[key]
            for i in f.out:
                if i != p:
                    orphans.append(i)
        fresh = [make(a, b, p) for (a, b) in horizon if (a * K + b) not in edges]
        assign(orphans, fresh)
        faces = [f for f in faces if f.alive] + fresh

    # Merge connected coplanar triangles into polygons (flood fill across shared edges).
    planes = []
    for f in faces:
        if f.group is not None:
            continue
        pl = {"n": f.n, "d": f.d, "ids": {}}
        f.group = pl
        stack = [f]
        while stack:
            g = stack.pop()
            for v in g.v:
                pl["ids"][v] = True
            for kk in range(3):
                nb = edges.get(g.v[(kk + 1) % 3] * K + g.v[kk])
                if (nb is not None and nb.group is None and _dot(nb.n, pl["n"]) > 0
                        and all(abs(_dot(pl["n"], P[v]) - pl["d"]) <= 10 * eps for v in nb.v)):
                    nb.group = pl
                    stack.append(nb)
        planes.append(pl)

    # Each face's boundary: 2-D convex hull of its points, counter-clockwise about the normal.
    loops = []
    for pl in planes:
        ids = list(pl["ids"].keys())
        c = [0.0, 0.0, 0.0]
        for i in ids:
            c = _add(c, P[i])
        c = _scale(c, 1.0 / len(ids))
        ref = [1.0, 0.0, 0.0] if abs(pl["n"][0]) < 0.9 else [0.0, 1.0, 0.0]
        u = _cross(pl["n"], ref)
        u = _scale(u, 1.0 / _norm(u))
        w = _cross(pl["n"], u)
        pts = [(i, _dot(_sub(P[i], c), u), _dot(_sub(P[i], c), w)) for i in ids]
        pts.sort(key=lambda q: (q[1], q[2]))

        def turn(o, a, b):
            return (a[1] - o[1]) * (b[2] - o[2]) - (a[2] - o[2]) * (b[1] - o[1])

        def half(lst):
            h = []
            for q in lst:
                while len(h) >= 2 and turn(h[-2], h[-1], q) <= eps * eps:
                    h.pop()
                h.append(q)
            h.pop()
            return h

        loop_ids = [q[0] for q in half(pts) + half(list(reversed(pts)))]
        if len(loop_ids) >= 3:
            loops.append({"n": pl["n"], "d": pl["d"], "ids": loop_ids})
    used = sorted({v for lp in loops for v in lp["ids"]})
    remap = {v: i for i, v in enumerate(used)}
    verts = [P[v] for v in used]
    out = [{"n": lp["n"], "d": lp["d"], "v": [remap[v] for v in lp["ids"]]} for lp in loops]
    return {"verts": verts, "faces": out}


def convex_hull_native(points):
    """``convex_hull`` computed by the library's C++ quickhull (``steel_convex_hull``; host only, no
    device needed): the same steps in the same order, so the same vertices, faces and planes, at a
    fraction of the cost. Raises ``SteelError`` where ``convex_hull`` raises ``ValueError``."""
    import ctypes

    from . import _lib
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    n = int(pts.shape[0])
    m = max(n, 1)
    verts = np.zeros(3 * m, np.float64)
    planes = np.zeros(8 * m, np.float64)
    start = np.zeros(2 * m + 1, np.uint32)
    fv = np.zeros(6 * m, np.uint32)
    nv, nf = ctypes.c_uint32(), ctypes.c_uint32()
    _lib.check(_lib.load().steel_convex_hull(pts.ctypes.data, n, verts.ctypes.data, planes.ctypes.data,
                                             start.ctypes.data, fv.ctypes.data, ctypes.byref(nv), ctypes.byref(nf)))
    V = verts[:3 * nv.value].reshape(-1, 3).tolist()
    faces = []
    for k in range(nf.value):
        pl = planes[4 * k:4 * k + 4].tolist()
        faces.append({"n": pl[:3], "d": pl[3], "v": fv[start[k]:start[k + 1]].astype(int).tolist()})
    return {"verts": V, "faces": faces}


def box_hull(h):
    """Hull of a box with half extents h, built directly: the 8 corners in shape_points order and
    6 quads counter-clockwise about their outward normals (planes n . x = d). Same solid as
    convex_hull(shape_points(BOX, h)) in a fixed vertex and face order, at a fraction of the cost."""
    verts = [[sx * h[0], sy * h[1], sz * h[2]] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]
    quads = [([1.0, 0.0, 0.0], h[0], [4, 6, 7, 5]), ([-1.0, 0.0, 0.0], h[0], [0, 1, 3, 2]),
             ([0.0, 1.0, 0.0], h[1], [2, 3, 7, 6]), ([0.0, -1.0, 0.0], h[1], [0, 4, 5, 1]),
             ([0.0, 0.0, 1.0], h[2], [1, 5, 7, 3]), ([0.0, 0.0, -1.0], h[2], [0, 2, 6, 4])]
    return {"verts": verts, "faces": [{"n": n, "d": float(d), "v": v} for n, d, v in quads]}


def shape_points(gtype, s):
    """Hull sample points of the analytic shapes (builder.js:176-196)."""
    pts = []
    if gtype == GT["BOX"]:
        for x in (-1, 1):
            for y in (-1, 1):
                for z in (-1, 1):
                    pts.append([x * s[0], y * s[1], z * s[2]])
    elif gtype == GT["CYLINDER"]:
        for z in (-s[1], s[1]):
            for i in range(24):
                a = (i * 2 * math.pi) / 24
                pts.append([s[0] * math.cos(a), s[0] * math.sin(a), z])
    elif gtype == GT["CAPSULE"]:
        for z0, sg in ((s[1], 1), (-s[1], -1)):
            for e in range(4):
                el = (e * math.pi) / 6
                for k in range(12):
                    az = (k * 2 * math.pi) / 12
                    pts.append([s[0] * math.cos(el) * math.cos(az), s[0] * math.cos(el) * math.sin(az),
                                z0 + sg * s[0] * math.sin(el)])
    elif gtype == GT["SPHERE"]:
        for e in range(7):
            el = -math.pi / 2 + (e * math.pi) / 6
            for k in range(12):
                az = (k * 2 * math.pi) / 12
                pts.append([s[0] * math.cos(el) * math.cos(az), s[0] * math.cos(el) * math.sin(az),
                            s[0] * math.sin(el)])
    return [[_js_round(v * 1e9) / 1e9 for v in p] for p in pts]


def mass_props(gtype, s, hull):
    """Unit-density mass, COM and inertia about the COM of a solid shape (builder.js:199-238)."""
    def diag(m, a, b, c):
        return {"m": m, "c": [0.0, 0.0, 0.0], "I": [a, 0.0, 0.0, 0.0, b, 0.0, 0.0, 0.0, c]}

    if gtype == GT["BOX"]:
        m = 8 * s[0] * s[1] * s[2]
        return diag(m, (m / 3) * (s[1] ** 2 + s[2] ** 2), (m / 3) * (s[0] ** 2 + s[2] ** 2),
                    (m / 3) * (s[0] ** 2 + s[1] ** 2))
    if gtype == GT["SPHERE"]:
        m = (4 / 3) * math.pi * s[0] ** 3
        i = 0.4 * m * s[0] ** 2
        return diag(m, i, i, i)
    if gtype == GT["CYLINDER"]:
        m = math.pi * s[0] ** 2 * 2 * s[1]
        t = m * (3 * s[0] ** 2 + 4 * s[1] ** 2) / 12
        return diag(m, t, t, 0.5 * m * s[0] ** 2)
    if gtype == GT["CAPSULE"]:
        r, L = s[0], 2 * s[1]
        mc, ms = math.pi * r * r * L, (4 / 3) * math.pi * r ** 3
        t = mc * (L * L / 12 + r * r / 4) + ms * (0.4 * r * r + L * L / 4 + 3 * L * r / 8)
        return diag(mc + ms, t, t, 0.5 * mc * r * r + 0.4 * ms * r * r)
    verts = hull["verts"]
    o = [0.0, 0.0, 0.0]
    for v in verts:
        o = _add(o, v)
    o = _scale(o, 1.0 / len(verts))
    m = 0.0
    c = [0.0, 0.0, 0.0]
    C = [0.0] * 9
    for f in hull["faces"]:
        for k in range(1, len(f["v"]) - 1):
            a = _sub(verts[f["v"][0]], o)
            b = _sub(verts[f["v"][k]], o)
            d = _sub(verts[f["v"][k + 1]], o)
            vol = _dot(a, _cross(b, d)) / 6
            m += vol
            c = _add(c, _scale(_add(_add(a, b), d), vol / 4))
            for i in range(3):
                for j in range(3):
                    C[i * 3 + j] += (vol / 20) * (2 * (a[i] * a[j] + b[i] * b[j] + d[i] * d[j]) + a[i] * b[j]
                                                  + a[j] * b[i] + a[i] * d[j] + a[j] * d[i] + b[i] * d[j] + b[j] * d[i])
    c = _scale(c, 1.0 / m)
    tr = C[0] + C[4] + C[8]
    I = [(tr if i == j else 0.0) - C[i * 3 + j] for i in range(3) for j in range(3)]
    for i in range(3):
        for j in range(3):
            I[i * 3 + j] -= m * ((_dot(c, c) if i == j else 0.0) - c[i] * c[j])
    return {"m": m, "c": _add(c, o), "I": I}


# --- loaded scene -------------------------------------------------------------------------
@dataclass
class LoadedScene:
    """The reference's ``LoadedScene`` (sceneTypes.ts:91-99): parsed scene.json plus scene.bin."""
    json: dict
    bin: bytes
    base: str = ""

    def f32(self, r) -> np.ndarray:
        return np.frombuffer(self.bin, dtype=np.float32, count=r["n"], offset=r["off"])

    def u32(self, r) -> np.ndarray:
        return np.frombuffer(self.bin, dtype=np.uint32, count=r["n"], offset=r["off"])


def load_scene(base: str) -> LoadedScene:
    """``loadScene`` (sim.js:40-61) for a scene folder on disk: scene.json + scene.bin."""
    import json
    import os
    with open(os.path.join(base, "scene.json")) as f:
        js = json.load(f)
    with open(os.path.join(base, "scene.bin"), "rb") as f:
        bn = f.read()
    return LoadedScene(js, bn, base)


# --- builder --------------------------------------------------------------------------------
_HULL_CACHE: dict = {}


def _hull_cached(gtype, size, pts, native=False):
    hull = convex_hull_native if native else convex_hull
    if pts is None:
        key = (gtype, tuple(size), native)
        h = _HULL_CACHE.get(key)
        if h is None:
            h = hull(shape_points(gtype, size))
            _HULL_CACHE[key] = h
        return h
    return hull(pts)


class SceneBuilder:
    """Newton-style ModelBuilder (builder.js:241-491). ``finalize()`` returns a ``LoadedScene``."""

    def __init__(self, gravity=(0.0, 0.0, -9.81), fps=60, box_hulls="quickhull", native_hulls=False):
        """box_hulls: "quickhull" (builder.js:264) or "direct" (box_hull, same solid, fixed order).
        native_hulls: compute hulls with the library's C++ quickhull (convex_hull_native)."""
        self.box_hulls = box_hulls
        self.native_hulls = native_hulls
        self.gravity = list(gravity)
        self.fps = fps
        self.bodies = []
        self.shapes = []
        self.joints = []
        self.filters = []
        self.dofOf = []

    def add_body(self, xform=IDENTITY, mass=None, com=None, inertia=None, label=None, kinematic=False,
                 gravity=True, twist=(0, 0, 0, 0, 0, 0)):
        self.bodies.append(dict(xform=[float(x) for x in xform], mass=mass, com=com, inertia=inertia,
                                label=label if label is not None else f"body_{len(self.bodies)}",
                                kinematic=kinematic, gravity=gravity, twist=[float(t) for t in twist]))
        return len(self.bodies) - 1

    def add_shape(self, body, gtype, size, opts=None, hull_points=None):
        o = dict(SHAPE_DEFAULTS)
        o.update(opts or {})
        if gtype == GT["PLANE"]:
            hull = None
        elif gtype == GT["BOX"] and hull_points is None and self.box_hulls == "direct":
            hull = box_hull([float(x) for x in size])
        else:
            hull = _hull_cached(gtype, size, hull_points, self.native_hulls)
        self.shapes.append(dict(body=body, type=gtype, size=list(size), xform=list(o.get("xform", IDENTITY)),
                                hull=hull, o=o))
        return len(self.shapes) - 1

    def add_shape_box(self, body, hx=0.5, hy=0.5, hz=0.5, **o):
        return self.add_shape(body, GT["BOX"], [hx, hy, hz], o)

    def add_shape_sphere(self, body, radius=0.5, **o):
        return self.add_shape(body, GT["SPHERE"], [radius, 0, 0], o)

    def add_shape_capsule(self, body, radius=0.05, half_height=0.5, **o):
        return self.add_shape(body, GT["CAPSULE"], [radius, half_height, 0], o)

    def add_shape_cylinder(self, body, radius=0.05, half_height=0.5, **o):
        return self.add_shape(body, GT["CYLINDER"], [radius, half_height, 0], o)

    def add_shape_convex_hull(self, body, vertices, **o):
        return self.add_shape(body, GT["CONVEX_MESH"], [1, 1, 1], o, [list(map(float, v)) for v in vertices])

    def add_ground_plane(self, height=0.0, **o):
        o = dict(o)
        o.setdefault("xform", [0.0, 0.0, height, 0.0, 0.0, 0.0, 1.0])
        return self.add_shape(-1, GT["PLANE"], [0, 0, 0], o)

    def add_collision_filter(self, a, b):
        self.filters.append((a, b))

    def add_joint(self, jtype, parent, child, parent_xform=IDENTITY, child_xform=IDENTITY, axes=(), linear=0,
                  q=None, label=None, collision_filter_parent=True, dofs=None, **dof):
        if dofs is None:
            dofs = []
            for _ in axes:
                d = dict(DOF_DEFAULTS)
                d.update(dof)
                dofs.append(d)
        self.joints.append(dict(type=jtype, parent=parent, child=child, Xp=list(parent_xform), Xc=list(child_xform),
                                axes=[list(a) for a in axes], linear=linear, q=q, label=label,
                                filter=collision_filter_parent, dofs=dofs, mimic=None))
        return len(self.joints) - 1

    def add_joint_revolute(self, parent, child, axis=(1, 0, 0), **o):
        return self.add_joint(JT["REVOLUTE"], parent, child, axes=[list(axis)], **o)

    def add_joint_prismatic(self, parent, child, axis=(1, 0, 0), **o):
        return self.add_joint(JT["PRISMATIC"], parent, child, axes=[list(axis)], linear=1, **o)

    def add_joint_ball(self, parent, child, **o):
        return self.add_joint(JT["BALL"], parent, child, axes=[[1, 0, 0], [0, 1, 0], [0, 0, 1]], **o)

    def add_joint_fixed(self, parent, child, **o):
        return self.add_joint(JT["FIXED"], parent, child, **o)

    def add_joint_d6(self, parent, child, linear_axes=(), angular_axes=(), parent_xform=IDENTITY,
                     child_xform=IDENTITY, q=None, label=None, collision_filter_parent=True, **shared):
        """D6 joint (builder.js:301-307): linear axes then angular axes, each [x, y, z] or dict(axis=..., **dof)."""
        entries = [e if isinstance(e, dict) else dict(axis=list(e)) for e in list(linear_axes) + list(angular_axes)]
        dofs = []
        for e in entries:
            d = dict(DOF_DEFAULTS)
            d.update(shared)
            d.update({k: v for k, v in e.items() if k != "axis"})
            dofs.append(d)
        return self.add_joint(JT["D6"], parent, child, parent_xform=parent_xform, child_xform=child_xform,
                              axes=[e["axis"] for e in entries], linear=len(linear_axes), q=q, label=label,
                              collision_filter_parent=collision_filter_parent, dofs=dofs)

    def add_joint_free(self, child, **o):
        return self.add_joint(JT["FREE"], -1, child,
                              axes=[[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], linear=3, **o)

    def set_joint_dof_config(self, joint, axis_index, **cfg):
        """Change dof settings of an existing joint, e.g. drive gains (builder.js:308-309)."""
        self.joints[joint]["dofs"][axis_index].update(cfg)

    def set_joint_mimic(self, joint, reference, coeffs=(0.0, 1.0)):
        """Newton's set_joint_mimic (builder.js:310-313): the joint's coordinates follow
        coeffs[0] + coeffs[1] * the reference joint's; reference None clears it."""
        self.joints[joint]["mimic"] = None if reference is None else dict(reference=reference, coeffs=list(coeffs))

    def joint_dof(self, joint):
        return self.dofOf[joint]

    def finalize(self, solver=None) -> LoadedScene:
        solver = solver or {}
        NB = len(self.bodies)
        parent_joint = [-1] * NB
        loop = []
        loop_set = set()
        for i, j in enumerate(self.joints):
            if j["child"] < 0 or j["child"] >= NB:
                raise ValueError(f"joint {i}: bad child body {j['child']}")
            if parent_joint[j["child"]] >= 0:
                loop.append(i)
                loop_set.add(i)
            else:
                parent_joint[j["child"]] = i
        order, art, implicit = [], [], []
        placed = set()

        def root_of(b):
            r, n = b, 0
            while parent_joint[r] >= 0 and self.joints[parent_joint[r]]["parent"] >= 0 and n < NB:
                n += 1
                r = self.joints[parent_joint[r]]["parent"]
            return r

        roots = sorted(set(root_of(b) for b in range(NB)))
        # Joints grouped by root body, in insertion order (one pass instead of a scan per root).
        by_root = {}
        for i, j in enumerate(self.joints):
            if i in loop_set:
                continue
            by_root.setdefault(root_of(j["child"]), []).append(i)
        order_set = set()
        for a, r in enumerate(roots):
            if parent_joint[r] < 0:
                implicit.append(dict(type=JT["FREE"], parent=-1, child=r, Xp=IDENTITY, Xc=IDENTITY,
                                     axes=[[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 0], [0, 1, 0], [0, 0, 1]],
                                     linear=3, label=f"{self.bodies[r]['label']}_free",
                                     dofs=[dict(DOF_DEFAULTS) for _ in range(6)], mimic=None, q=None))
                order.append(-len(implicit))
                art.append(a)
            for i in by_root.get(r, []):
                j = self.joints[i]
                if (j["parent"] >= 0 and j["parent"] not in placed and root_of(j["parent"]) == r
                        and parent_joint[j["parent"]] >= 0 and parent_joint[j["parent"]] not in order_set):
                    raise ValueError(f"joint {i}: add the joint of parent body {j['parent']} before its children")
                order.append(i)
                order_set.add(i)
                art.append(a)
                placed.add(j["child"])
            placed.add(r)
        for i in loop:
            order.append(i)
            art.append(-1)

        def joint_at(k):
            return implicit[-k - 1] if k < 0 else self.joints[k]

        J = dict(type=[], parent=[], child=[], X_p=[], X_c=[], axis=[], dof_dim=[], q_start=[0], qd_start=[0],
                 articulation=art, q=[], qd=[], armature=[], ke=[], kd=[], effort=[], lower=[], upper=[],
                 vel_limit=[], friction=[], passive_damping=[], target_q=[], target_qd=[], mimic_joint=[],
                 mimic_coeffs=[], friction_load_coefficient=[], label=[])
        self.dofOf = [0] * len(self.joints)
        for idx, k in enumerate(order):
            j = joint_at(k)
            if k >= 0:
                self.dofOf[k] = J["qd_start"][idx]
            ndof = len(j["axes"])
            scalar = j["type"] in (JT["REVOLUTE"], JT["PRISMATIC"], JT["D6"])
            if j["type"] == JT["FREE"]:
                q = list(self.bodies[j["child"]]["xform"])
            elif j["type"] == JT["BALL"]:
                q = list(j.get("q") or [0.0, 0.0, 0.0, 1.0])
            elif scalar:
                q0 = j.get("q")
                q0 = [0.0] if q0 is None else (list(q0) if isinstance(q0, (list, tuple)) else [q0])
                q = (q0 + [0.0] * ndof)[:ndof]
            else:
                q = []
            J["type"].append(j["type"])
            J["parent"].append(j["parent"])
            J["child"].append(j["child"])
            J["X_p"].append(list(j["Xp"]))
            J["X_c"].append(list(j["Xc"]))
            J["dof_dim"].append([j["linear"], ndof - j["linear"]])
            J["q"].extend(q)
            J["target_q"].extend([d["targetPos"] for d in j["dofs"]] if scalar else [0.0] * len(q))
            J["q_start"].append(len(J["q"]))
            J["qd"].extend(self.bodies[j["child"]]["twist"] if j["type"] == JT["FREE"] else [0.0] * ndof)
            for a_i, ax in enumerate(j["axes"]):
                d = j["dofs"][a_i]
                J["axis"].append(list(ax))
                J["armature"].append(d["armature"])
                J["ke"].append(d["targetKe"])
                J["kd"].append(d["targetKd"])
                J["effort"].append(d["effortLimit"])
                J["lower"].append(d["limitLower"])
                J["upper"].append(d["limitUpper"])
                J["vel_limit"].append(d["velocityLimit"])
                J["friction"].append(d["friction"])
                J["passive_damping"].append(d["damping"])
                J["target_qd"].append(d["targetVel"])
            J["qd_start"].append(len(J["axis"]))
            J["mimic_joint"].append(-1)
            J["mimic_coeffs"].append(list(j["mimic"]["coeffs"]) if j.get("mimic") else [0, 1])
            J["label"].append(j.get("label") or f"joint_{idx}")
        J["count"] = len(order)
        final_index = {k: idx for idx, k in enumerate(order)}
        for idx, k in enumerate(order):
            m = joint_at(k).get("mimic")
            if m:
                J["mimic_joint"][idx] = final_index[m["reference"]]

        # Forward kinematics for the initial body poses (builder.js:390-413).
        pose = [list(b["xform"]) for b in self.bodies]
        for idx, k in enumerate(order):
            if art[idx] < 0:
                continue
            j = joint_at(k)
            if j["type"] == JT["FREE"]:
                continue
            qs = J["q_start"][idx]
            T = list(IDENTITY)
            if j["type"] == JT["REVOLUTE"]:
                T = [0.0, 0.0, 0.0] + qaxis(j["axes"][0], J["q"][qs])
            elif j["type"] == JT["PRISMATIC"]:
                T = _scale(j["axes"][0], J["q"][qs] / _norm(j["axes"][0])) + [0.0, 0.0, 0.0, 1.0]
            elif j["type"] == JT["BALL"]:
                T = [0.0, 0.0, 0.0] + J["q"][qs:qs + 4]
            elif j["type"] == JT["D6"]:
                p = [0.0, 0.0, 0.0]
                r = [0.0, 0.0, 0.0, 1.0]
                for a_i in range(j["linear"]):
                    p = _add(p, _scale(j["axes"][a_i], J["q"][qs + a_i]))
                for a_i in range(j["linear"], len(j["axes"])):
                    ax = qrot(r, _scale(j["axes"][a_i], 1.0 / _norm(j["axes"][a_i])))
                    r = qmul(qaxis(ax, J["q"][qs + a_i]), r)
                T = p + r
            Xwp = pose[j["parent"]] if j["parent"] >= 0 else IDENTITY
            pose[j["child"]] = tmul(tmul(tmul(Xwp, j["Xp"]), T), tinv(j["Xc"]))

        # Mass properties from the shapes unless given (builder.js:415-444).
        bodies = dict(count=NB, mass=[], inertia=[], com=[], q=pose, twist=[], label=[], kinematic=[], no_gravity=[])
        shapes_by_body = {}
        for s in self.shapes:
            shapes_by_body.setdefault(s["body"], []).append(s)
        for i, b in enumerate(self.bodies):
            m = 0.0
            c = [0.0, 0.0, 0.0]
            parts = []
            for s in shapes_by_body.get(i, []):
                if s["type"] == GT["PLANE"] or not ((s["o"].get("mass") or 0) > 0 or (s["o"].get("density") or 0) > 0):
                    continue
                p = mass_props(s["type"], s["size"], s["hull"])
                rho = s["o"]["mass"] / p["m"] if (s["o"].get("mass") or 0) > 0 else s["o"]["density"]
                pm = p["m"] * rho
                pc = _add(s["xform"][:3], qrot(s["xform"][3:], p["c"]))
                parts.append(dict(m=pm, c=pc, I=[v * rho for v in p["I"]], R=qmat(s["xform"][3:])))
                m += pm
                c = _add(c, _scale(pc, pm))
            c = _scale(c, 1.0 / m) if m > 0 else [0.0, 0.0, 0.0]
            I = [0.0] * 9
            for p in parts:
                d = _sub(p["c"], c)
                for r in range(3):
                    for s_ in range(3):
                        v = 0.0
                        for a_ in range(3):
                            for e_ in range(3):
                                v += p["R"][r * 3 + a_] * p["I"][a_ * 3 + e_] * p["R"][s_ * 3 + e_]
                        I[r * 3 + s_] += v + p["m"] * ((_dot(d, d) if r == s_ else 0.0) - d[r] * d[s_])
            bodies["mass"].append(b["mass"] if b["mass"] is not None else m)
            bodies["com"].append(b["com"] if b["com"] is not None else c)
            if b["inertia"] is not None:
                bodies["inertia"].append(b["inertia"])
            elif b["mass"] is not None and m > 0:
                bodies["inertia"].append([v * b["mass"] / m for v in I])
            else:
                bodies["inertia"].append(I)
            bodies["twist"].append(b["twist"])
            bodies["label"].append(b["label"])
            bodies["kinematic"].append(b["kinematic"])
            bodies["no_gravity"].append(not b["gravity"])

        # Binary blob: hull geometry (builder.js:446-468).
        chunks = []
        size = [0]

        def put(arr: np.ndarray):
            off = size[0]
            chunks.append(arr.tobytes())
            size[0] += arr.nbytes
            return {"off": off, "n": int(arr.size)}

        shapes = []
        index = {}
        hull_refs = {}
        for sid, s in enumerate(self.shapes):
            o = s["o"]
            entry = dict(sid=sid, body=s["body"], xf=list(s["xform"]), type=s["type"], color=o["color"], mu=o["mu"],
                         gap=o["gap"], restitution=o["restitution"], mu_torsional=o["muTorsional"],
                         mu_rolling=o["muRolling"], group=o["collisionGroup"], condim=3, ke=o["ke"], kd=o["kd"],
                         torsion_radius=0, world=o["world"])
            if s["type"] == GT["PLANE"]:
                entry["plane"] = True
            else:
                h = s["hull"]
                # Identical hull objects share one blob range (the packer dedups hulls by verts offset).
                ref = hull_refs.get(id(h))
                if ref is None:
                    fv, fstart, fn = [], [], []
                    for f in h["faces"]:
                        fstart.append(len(fv))
                        fv.extend(f["v"])
                        fn.extend(list(f["n"]) + [f["d"]])
                    ref = dict(verts=put(np.asarray(h["verts"], dtype=np.float32).reshape(-1)),
                               face_planes=put(np.asarray(fn, dtype=np.float32)),
                               face_start=put(np.asarray(fstart + [len(fv)], dtype=np.uint32)),
                               face_verts=put(np.asarray(fv, dtype=np.uint32)),
                               nv=len(h["verts"]), nf=len(h["faces"]))
                    hull_refs[id(h)] = ref
                entry["hull"] = ref
                if s["type"] == GT["SPHERE"]:
                    entry["prim"] = dict(kind=1, r=s["size"][0], h=0)
                if s["type"] == GT["CAPSULE"]:
                    entry["prim"] = dict(kind=2, r=s["size"][0], h=s["size"][1])
            index[sid] = len(shapes)
            shapes.append(entry)
        # Newton's collision_filter_parent: a joint's two bodies do not collide (builder.js:470-477).
        pairs = {}
        for a, b in self.filters:
            pairs[(min(a, b), max(a, b))] = True
        shape_ids_by_body = {}
        for i, s_ in enumerate(self.shapes):
            shape_ids_by_body.setdefault(s_["body"], []).append(i)
        for j in self.joints:
            if not j["filter"] or j["parent"] < 0:
                continue
            pa = shape_ids_by_body.get(j["parent"], [])
            ch = shape_ids_by_body.get(j["child"], [])
            for a in pa:
                for b in ch:
                    if a != b:
                        pairs[(min(a, b), max(a, b))] = True
        targets = put(np.zeros(0, dtype=np.float32))
        bin_ = b"".join(chunks)
        s = dict(substeps=4, iterations=12, enable_joint_limits=True)
        s.update(solver)
        js = dict(gravity=list(self.gravity), fps=self.fps, substeps=s["substeps"], iterations=s["iterations"],
                  bodies=bodies, joints=J, shapes=shapes, visuals=[],
                  filters=[[index[a], index[b]] for (a, b) in pairs.keys()],
                  mimics=[], targets=targets, target_frames=0, driven=0, integral_count=0, demo="built",
                  control=None, solver=s, info={}, joint_type_names=dict(JT), geo_type_names=dict(GT))
        return LoadedScene(js, bin_)
