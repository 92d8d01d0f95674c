"""Scene packing: the reference's ``Sim.build()`` restated in Python.

Follows ``packages/steel-webgpu/src/sim.js:95-521``: articulation and dof tables
(sim.js:99-157), mimics (sim.js:160-172), hull dedup and unique edges
(sim.js:180-209), the ``statF``/``statU`` static buffers (sim.js:212-393),
capacities and solver flags (sim.js:395-477), the per-substep parameter block
(``writeParams``, sim.js:625-639) and the initial state (sim.js:486-502).

The output is the reference's own static format: ``statF`` is an array of
vec4 (float32), ``statU`` an array of u32, and ``C`` the dictionary of
compile-time constants the reference bakes into its WGSL (sim.js:456-477).
The CUDA library takes exactly this (plus the initial state) across its C ABI,
the way the reference hands it to ``device.queue.writeBuffer``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .builder import JT, LoadedScene

COMBINE = ["average", "min", "multiply", "max"]
LB = 268          # floats per link block (artwgsl.js:8)
L_V = 147         # link record: spatial velocity (artwgsl.js:15)
MAX_SUBSTEPS = 32


def _f32(x) -> float:
    return float(np.float32(x))


def quat_rotate(q, v):
    """sim.js:16-22 (double precision)."""
    x, y, z, w = q
    ux = 2 * (x * v[0] + y * v[1] + z * v[2])
    s2 = w * w - (x * x + y * y + z * z)
    cx, cy, cz = y * v[2] - z * v[1], z * v[0] - x * v[2], x * v[1] - y * v[0]
    return [ux * x + s2 * v[0] + 2 * w * cx, ux * y + s2 * v[1] + 2 * w * cy, ux * z + s2 * v[2] + 2 * w * cz]


def inv3(m):
    """sim.js:24-31."""
    a, b, c, d, e, f, g, h, i = m
    A = e * i - f * h
    B = -(d * i - f * g)
    C = d * h - e * g
    det = a * A + b * B + c * C
    if abs(det) < 1e-30:
        return [0.0] * 9
    k = 1 / det
    return [A * k, -(b * i - c * h) * k, (b * f - c * e) * k, B * k, (a * i - c * g) * k, -(a * f - c * d) * k,
            C * k, -(a * h - b * g) * k, (a * e - b * d) * k]


@dataclass
class Packed:
    """One packed scene: the reference's static buffers, constants and initial state."""
    C: dict
    statF: np.ndarray           # float32, length = 4 * vec4 count
    statU: np.ndarray           # uint32
    body_pose: np.ndarray       # float32, NB * 8 (COM xyz, 0, quat xyzw)
    body_vel: np.ndarray        # float32, NB * 8 (v xyz, 0, w xyz, 0)
    art: np.ndarray             # float32, art buffer initial contents (A_* layout)
    params: dict                # inputs of writeParams (sim.js:625-639)
    links: list
    dof_map: dict               # Newton dof -> port dof
    q_map: dict                 # Newton coordinate -> port coordinate
    body_kind: list
    NB: int
    NS: int
    NA: int
    NL: int
    ND: int
    NQ: int
    joints: dict                # the scene's joint arrays (for state())
    body_com: list
    layout: dict = field(default_factory=dict)

    def constants_text(self) -> str:
        """``KEY=VALUE`` lines: the reference's C plus the writeParams inputs (prefixed ``PARAM_``)."""
        lines = []
        for k, v in self.C.items():
            lines.append(f"{k}={_fmt(v)}")
        for k, v in self.params.items():
            if isinstance(v, (list, tuple)):
                for i, x in enumerate(v):
                    lines.append(f"PARAM_{k}{i}={_fmt(x)}")
            else:
                lines.append(f"PARAM_{k}={_fmt(v)}")
        return "\n".join(lines) + "\n"


def _fmt(v) -> str:
    if isinstance(v, bool):
        return "1" if v else "0"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def pack(scene: LoadedScene, opts: dict | None = None, colorWords: int | None = None,
         caps: dict | None = None) -> Packed:
    """``Sim.build()`` (sim.js:95-521) without the WebGPU calls.

    ``caps`` optionally overrides the reference's fixed capacities (MAXP, MAXC, MAXU, UH, WH,
    MAXDENSE, AH): the defaults are the reference's; results only depend on them when a
    capacity overflows.
    """
    S = scene.json
    given = {k: v for k, v in (opts or {}).items() if v is not None}
    o = dict(substeps=S["substeps"], iterations=S["iterations"],
             regularization=(S.get("solver") or {}).get("contact_regularization", 0.0) or 0.0)
    if (S.get("solver") or {}).get("contact_regularization") is None:
        o["regularization"] = 0.0
    o.update(given)
    if o["substeps"] > MAX_SUBSTEPS:
        raise ValueError(f"at most {MAX_SUBSTEPS} substeps")
    f32 = scene.f32
    u32 = scene.u32
    NB = S["bodies"]["count"]
    J = S["joints"]
    bodies = S["bodies"]
    kin = bodies.get("kinematic") or []

    def is_kin(b):
        return bool(kin[b]) if b < len(kin) else False

    joint_of_body = [-1] * NB
    for j in range(J["count"]):
        joint_of_body[J["child"][j]] = j
    art_joints: dict = {}
    for j in range(J["count"]):
        art_joints.setdefault(J["articulation"][j], []).append(j)
    body_kind = [1] * NB
    body_art = [-1] * NB
    body_link = [-1] * NB
    arts, links, dofs = [], [], []
    SO = dict(S.get("solver") or {})
    SO.update(o.get("solver") or {})
    limits_on = SO.get("enable_joint_limits", False) or False
    q0, tq0, tqd0 = [], [], []
    q_map, dof_map = {}, {}
    loops = []
    for art, js in art_joints.items():
        if art < 0:
            loops.extend(js)
            continue
        if len(js) == 1 and J["type"][js[0]] in (JT["FREE"], JT["DISTANCE"]):
            continue
        a = len(arts)
        link_start, dof_start = len(links), len(dofs)
        local_link = {}
        for j in js:
            t = JT["FREE"] if J["type"][j] == JT["DISTANCE"] else J["type"][j]
            b = J["child"][j]
            l = len(links)
            local_link[b] = l
            parent_link = local_link.get(J["parent"][j], None) if J["parent"][j] >= 0 else -1
            if parent_link is None:
                parent_link = -1
            if t not in (JT["FIXED"], JT["REVOLUTE"], JT["PRISMATIC"], JT["BALL"], JT["FREE"], JT["D6"]):
                raise ValueError(f"joint type {t} is not supported yet")
            ndof = J["qd_start"][j + 1] - J["qd_start"][j]
            nq = J["q_start"][j + 1] - J["q_start"][j]
            dof, qs = len(dofs), len(q0)
            scalar = t in (JT["REVOLUTE"], JT["PRISMATIC"], JT["D6"])
            for k in range(ndof):
                qd = J["qd_start"][j] + k
                limited = bool(limits_on and scalar and J["lower"][qd] > -1e5 and J["upper"][qd] < 1e5)
                friction = J["friction"][qd] if SO.get("enable_joint_friction") else 0.0
                pdmp = J.get("passive_damping")
                spk = J.get("spring_stiffness")
                spr = J.get("spring_ref")
                flc = J.get("friction_load_coefficient")
                dofs.append(dict(
                    armature=1e9 if is_kin(J["child"][j]) else J["armature"][qd], ke=J["ke"][qd], kd=J["kd"][qd],
                    effort=J["effort"][qd], lower=J["lower"][qd], upper=J["upper"][qd], limited=1 if limited else 0,
                    link=len(links), damping=(pdmp[qd] if pdmp and qd < len(pdmp) and pdmp[qd] is not None else 0.0),
                    friction=friction, axis=J["axis"][qd], scalar=scalar,
                    springKe=(spk[qd] if (scalar and spk and qd < len(spk) and spk[qd] is not None) else 0.0),
                    springRef=(spr[qd] if spr and qd < len(spr) and spr[qd] is not None else 0.0),
                    loadCoef=((flc[qd] if flc and qd < len(flc) and flc[qd] is not None else 0.0)
                              if (SO.get("enable_joint_friction") and scalar) else 0.0),
                    velLimit=(J["vel_limit"][qd] if (scalar and SO.get("enable_joint_velocity_limits")
                                                    and J["vel_limit"][qd] < 1e5) else -1.0)))
                tqd = J.get("target_qd")
                tqd0.append(tqd[qd] if tqd else 0.0)
            for k in range(nq):
                q_map[J["q_start"][j] + k] = len(q0)
                q0.append(J["q"][J["q_start"][j] + k])
            for k in range(ndof):
                dof_map[J["qd_start"][j] + k] = dof + k
            tq_src = J.get("target_q") or J["q"]
            for k in range(ndof):
                tq0.append(tq_src[J["q_start"][j] + k] if scalar else 0.0)
            parent_movable = parent_link >= 0 and links[parent_link]["movable"]
            dd = J.get("dof_dim")
            nlin = (dd[j][0] if dd and j < len(dd) and dd[j] else 0) or 0
            links.append(dict(type=t, parent=parent_link, dof=dof, ndof=ndof, nlin=nlin, qs=qs, body=b, joint=j,
                              movable=ndof > 0 or parent_movable))
            body_kind[b] = 2
            body_art[b] = a
            body_link[b] = l
        arts.append(dict(linkStart=link_start, linkCount=len(links) - link_start, dofStart=dof_start,
                         dofCount=len(dofs) - dof_start))
    NA, NL, ND = len(arts), len(links), len(dofs)
    mimics = []

    def add_mimic(f, r, c0, c1):
        n = J["qd_start"][f + 1] - J["qd_start"][f]
        for k in range(n):
            fd = dof_map.get(J["qd_start"][f] + k)
            ld = dof_map.get(J["qd_start"][r] + k)
            a_ = body_art[J["child"][f]]
            if fd is None or ld is None or a_ != body_art[J["child"][r]]:
                raise ValueError("mimic joints must share an articulation")
            d0 = arts[a_]["dofStart"]
            mimics.append(dict(art=a_, f=fd - d0, l=ld - d0, c0=c0, c1=c1, fq=q_map[J["q_start"][f] + k],
                               lq=q_map[J["q_start"][r] + k]))

    for f, r in enumerate(J.get("mimic_joint") or []):
        if r >= 0:
            add_mimic(f, r, J["mimic_coeffs"][f][0], J["mimic_coeffs"][f][1])
    for m in S.get("mimics") or []:
        if m.get("enabled"):
            add_mimic(m["follower"], m["leader"], m["c0"], m["c1"])

    # Hulls (sim.js:180-209).
    hull_index = {}
    hulls = []
    shapes = [s for s in S["shapes"] if s.get("hull") or s.get("plane")]
    for s in shapes:
        if not s.get("hull"):
            continue
        key = s["hull"]["verts"]["off"]
        if key not in hull_index:
            hull_index[key] = len(hulls)
            hulls.append(s["hull"])
    NS, NH = len(shapes), len(hulls)
    n_verts = sum(h["nv"] for h in hulls)
    n_faces = sum(h["nf"] for h in hulls)
    n_fv = sum(h["face_verts"]["n"] for h in hulls)
    hull_edges = []
    for h in hulls:
        fs = u32(h["face_start"])
        fv = u32(h["face_verts"])
        faces = {}
        edges = []
        for f in range(h["nf"]):
            n = int(fs[f + 1] - fs[f])
            for i in range(n):
                a_, b_ = int(fv[fs[f] + i]), int(fv[fs[f] + (i + 1) % n])
                key = min(a_, b_) * 65536 + max(a_, b_)
                faces.setdefault(key, []).append(f)
                if a_ < b_:
                    edges.append((a_, b_, key))
        hull_edges.append([(a_, b_, faces[key][0], faces[key][-1]) for (a_, b_, key) in edges])
    n_edges = sum(len(e) for e in hull_edges)
    path_floats = S.get("target_frames", 0) * S.get("driven", 0)

    SF = {}
    off = 0
    for k, n in (("SF_BODY", NB * 8), ("SF_SHAPE", NS * 7), ("SF_HAABB", NH * 2), ("SF_VERTS", n_verts),
                 ("SF_FPLANE", n_faces), ("SF_LINK", max(NL, 1) * 6), ("SF_DOF", max(ND, 1) * 5),
                 ("SF_PATH", math.ceil(path_floats / 4)), ("SF_LOOP", max(len(loops), 1) * 5),
                 ("SF_MIMIC", max(len(mimics), 1) * 2), ("SF_CTRL", 1)):
        SF[k] = off
        off += n
    statF = np.zeros(off * 4, dtype=np.float32)
    SU = {}
    uoff = 0
    for k, n in (("SU_HULL", NH * 4), ("SU_FACE", n_faces * 2), ("SU_FV", n_fv), ("SU_HEDGE", NH * 2),
                 ("SU_EDGE", n_edges * 4), ("SU_ART", max(NA, 1) * 4), ("SU_ACON", max(NA, 1)),
                 ("SU_FILTER", math.ceil((NS * NS) / 32))):
        SU[k] = uoff
        uoff += n
    statU = np.zeros(uoff, dtype=np.uint32)

    # Collision filter bitset (sim.js:235-255), vectorised over the NS x NS matrix.
    index = {}
    for i, sh in enumerate(S["shapes"]):
        if sh.get("hull") or sh.get("plane"):
            index[i] = len(index)
    filt = np.zeros((NS, NS), dtype=bool)
    for a0, b0 in S.get("filters") or []:
        a_, b_ = index.get(a0), index.get(b0)
        if a_ is None or b_ is None:
            continue
        filt[a_, b_] = True
        filt[b_, a_] = True
    worlds = np.array([(sh.get("world") if sh.get("world") is not None else -1) for sh in shapes], dtype=np.int64)
    groups = np.array([(sh.get("group") if sh.get("group") is not None else -1) for sh in shapes], dtype=np.int64)
    if NS:
        wa, wb = worlds[:, None], worlds[None, :]
        ga, gb = groups[:, None], groups[None, :]
        groups_meet = (ga != 0) & (gb != 0) & np.where(ga > 0, (ga == gb) | (gb < 0), ga != gb)
        meet = ((wa < 0) | (wb < 0) | (wa == wb)) & groups_meet
        upper = np.triu(np.ones((NS, NS), dtype=bool), 1)
        bad = upper & ~meet
        filt |= bad | bad.T
        bits = np.zeros(SU and (uoff - SU["SU_FILTER"]) * 32, dtype=bool)
        bits[:NS * NS] = filt.reshape(-1)
        words = np.packbits(bits.reshape(-1, 8), axis=1, bitorder="little").reshape(-1).view("<u4")
        statU[SU["SU_FILTER"]:SU["SU_FILTER"] + words.size] = words

    # Bodies (sim.js:257-305).
    body_pose = np.zeros(NB * 8, dtype=np.float32)
    sf = statF
    for b in range(NB):
        o_ = (SF["SF_BODY"] + b * 8) * 4
        m = bodies["mass"][b]
        link = body_link[b]
        kind = 3 if (body_kind[b] == 2 and not links[link]["movable"]) else body_kind[b]
        body_kind[b] = kind
        kinematic = is_kin(b)
        sf[o_] = (1 / m) if (m > 0 and not kinematic) else 0.0
        sf[o_ + 1] = kind
        sf[o_ + 2] = body_art[b]
        sf[o_ + 3] = link
        com = bodies["com"][b]
        sf[o_ + 4:o_ + 8] = [com[0], com[1], com[2], max(m, 0)]
        I = bodies["inertia"][b]
        Ii = inv3(I)
        for r in range(3):
            sf[o_ + 8 + r * 4:o_ + 12 + r * 4] = [I[r * 3], I[r * 3 + 1], I[r * 3 + 2], 0]
            sf[o_ + 20 + r * 4:o_ + 24 + r * 4] = ([0, 0, 0, 0] if kinematic else
                                                   [Ii[r * 3], Ii[r * 3 + 1], Ii[r * 3 + 2], 0])
        bq = bodies["q"][b]
        q = [bq[3], bq[4], bq[5], bq[6]]
        c = quat_rotate(q, com)
        body_pose[b * 8:b * 8 + 8] = [bq[0] + c[0], bq[1] + c[1], bq[2] + c[2], 0, *q]
    radius = np.zeros(NB, dtype=np.float32)
    for s in shapes:
        if s["body"] < 0 or s.get("plane"):
            continue
        com = bodies["com"][s["body"]]
        prim = s.get("prim") or {}
        pk = prim.get("kind", 0)
        sr = prim["r"] if pk == 1 else (prim["r"] + prim["h"] if pk == 2 else 0.0)
        if s.get("hull") and not pk:
            v = f32(s["hull"]["verts"]).astype(np.float64)
            for i in range(s["hull"]["nv"]):
                sr = max(sr, math.hypot(v[i * 3], v[i * 3 + 1], v[i * 3 + 2]))
        d = math.hypot(s["xf"][0] - com[0], s["xf"][1] - com[1], s["xf"][2] - com[2])
        radius[s["body"]] = max(radius[s["body"]], np.float32(d + sr))
    no_grav = bodies.get("no_gravity") or []
    for b in range(NB):
        o_ = (SF["SF_BODY"] + b * 8) * 4
        sf[o_ + 11] = radius[b]
        sf[o_ + 31] = (1 if is_kin(b) else 0) | (2 if (b < len(no_grav) and no_grav[b]) else 0)

        def lim(k):
            arr = bodies.get(k)
            if arr is None or b >= len(arr) or arr[b] is None:
                return -1.0
            return arr[b]

        ad = bodies.get("angular_damping")
        sf[o_ + 15] = ad[b] if (ad is not None and b < len(ad) and ad[b] is not None) else 0.05
        sf[o_ + 19] = lim("max_linear_velocity")
        sf[o_ + 23] = lim("max_angular_velocity")
        sf[o_ + 27] = lim("max_depenetration_velocity")

    # Reduction groups (sim.js:306-313).
    rkeys = {}
    rgroup = []
    for i, s in enumerate(shapes):
        if s["body"] < 0:
            k = ("s", i)
        else:
            k = (s["body"], s.get("mu"), s.get("restitution"), s.get("mu_torsional"), s.get("mu_rolling"),
                 s.get("ke"), s.get("kd"), s.get("condim"), s.get("torsion_radius"))
        if k not in rkeys:
            rkeys[k] = len(rkeys)
        rgroup.append(rkeys[k])
    GTn = S["geo_type_names"]

    def geo_scale(s):
        if s["type"] in (GTn["SPHERE"], GTn["CAPSULE"]):
            return [s["prim"]["r"], s["prim"]["h"], 0]
        if s["type"] not in (GTn["BOX"], GTn["CYLINDER"]):
            return [1, 1, 1]
        v = f32(s["hull"]["verts"])
        m = [0.0, 0.0, 0.0]
        for i in range(v.size):
            m[i % 3] = max(m[i % 3], abs(float(v[i])))
        return m if s["type"] == GTn["BOX"] else [m[0], m[2], 0]

    for i, s in enumerate(shapes):
        o_ = (SF["SF_SHAPE"] + i * 7) * 4
        prim = s.get("prim") or {}
        sf[o_:o_ + 4] = [s["body"], hull_index[s["hull"]["verts"]["off"]] if s.get("hull") else 0, s["mu"],
                         s["gap"] if s.get("gap") is not None else 0.001]
        xf = s["xf"]
        sf[o_ + 4:o_ + 12] = [xf[0], xf[1], xf[2], 0, xf[3], xf[4], xf[5], xf[6]]
        sf[o_ + 20:o_ + 24] = [s.get("ke") or 0, s.get("kd") or 0, rgroup[i], 0]
        sf[o_ + 12:o_ + 16] = [4 if s.get("plane") else prim.get("kind", 0), prim.get("r", 0), prim.get("h", 0),
                               s.get("torsion_radius") or 0]
        sf[o_ + 16:o_ + 20] = [s.get("restitution") or 0, s.get("mu_torsional") or 0, s.get("mu_rolling") or 0,
                               s.get("condim") if s.get("condim") is not None else 3]
        sf[o_ + 24:o_ + 28] = [GTn["PLANE"] if s.get("plane") else s["type"], *geo_scale(s)]

    # Hull geometry (sim.js:334-355).
    v_off = f_off = fv_off = e_off = 0
    for hi, h in enumerate(hulls):
        statU[SU["SU_HEDGE"] + hi * 2:SU["SU_HEDGE"] + hi * 2 + 2] = [e_off, len(hull_edges[hi])]
        for k, e in enumerate(hull_edges[hi]):
            statU[SU["SU_EDGE"] + (e_off + k) * 4:SU["SU_EDGE"] + (e_off + k) * 4 + 4] = e
        e_off += len(hull_edges[hi])
        v = f32(h["verts"])
        planes = f32(h["face_planes"])
        fs = u32(h["face_start"])
        fv = u32(h["face_verts"])
        vv = v.reshape(-1, 3).astype(np.float64)
        lo = vv.min(axis=0)
        hiB = vv.max(axis=0)
        base = (SF["SF_VERTS"] + v_off) * 4
        vert4 = np.zeros((h["nv"], 4), dtype=np.float32)
        vert4[:, :3] = v.reshape(-1, 3)
        sf[base:base + h["nv"] * 4] = vert4.reshape(-1)
        sf[(SF["SF_HAABB"] + hi * 2) * 4:(SF["SF_HAABB"] + hi * 2) * 4 + 8] = [
            (lo[0] + hiB[0]) / 2, (lo[1] + hiB[1]) / 2, (lo[2] + hiB[2]) / 2, 0,
            (hiB[0] - lo[0]) / 2, (hiB[1] - lo[1]) / 2, (hiB[2] - lo[2]) / 2, 0]
        statU[SU["SU_HULL"] + hi * 4:SU["SU_HULL"] + hi * 4 + 4] = [v_off, h["nv"], f_off, h["nf"]]
        for f in range(h["nf"]):
            sf[(SF["SF_FPLANE"] + f_off + f) * 4:(SF["SF_FPLANE"] + f_off + f) * 4 + 4] = planes[f * 4:f * 4 + 4]
            statU[SU["SU_FACE"] + (f_off + f) * 2:SU["SU_FACE"] + (f_off + f) * 2 + 2] = [fv_off + int(fs[f]),
                                                                                         int(fs[f + 1] - fs[f])]
        statU[SU["SU_FV"] + fv_off:SU["SU_FV"] + fv_off + fv.size] = fv
        v_off += h["nv"]
        f_off += h["nf"]
        fv_off += fv.size

    # Articulations (sim.js:356-393).
    for i, l in enumerate(links):
        o_ = (SF["SF_LINK"] + i * 6) * 4
        xp, xc = J["X_p"][l["joint"]], J["X_c"][l["joint"]]
        ax = J["axis"][J["qd_start"][l["joint"]]] if l["ndof"] == 1 else [0, 0, 1]
        sf[o_:o_ + 24] = [l["type"], l["parent"], l["dof"], l["body"],
                          xp[0], xp[1], xp[2], l["ndof"], xp[3], xp[4], xp[5], xp[6],
                          xc[0], xc[1], xc[2], l["qs"], xc[3], xc[4], xc[5], xc[6],
                          ax[0], ax[1], ax[2], l["nlin"] if l["type"] == JT["D6"] else 0]
    for i, d in enumerate(dofs):
        o_ = (SF["SF_DOF"] + i * 5) * 4
        sf[o_:o_ + 20] = [d["armature"], d["ke"], d["kd"], d["effort"], d["lower"], d["upper"], d["limited"],
                          d["link"], d["damping"], d["friction"], d["velLimit"], 1 if d["scalar"] else 0,
                          d["axis"][0], d["axis"][1], d["axis"][2], d["loadCoef"], d["springKe"], d["springRef"],
                          0, 0]
    for i, a_ in enumerate(arts):
        statU[SU["SU_ART"] + i * 4:SU["SU_ART"] + i * 4 + 4] = [a_["linkStart"], a_["linkCount"], a_["dofStart"],
                                                               a_["dofCount"]]
    for m in mimics:
        statU[SU["SU_ACON"] + m["art"]] = 1
    for j in loops:
        statU[SU["SU_ACON"] + body_art[J["child"][j]]] = 1
    tg = S.get("targets")
    if tg and tg.get("n", 0):
        tv = f32(tg)
        sf[SF["SF_PATH"] * 4:SF["SF_PATH"] * 4 + tv.size] = tv
    for i, j in enumerate(loops):
        t = J["type"][j]
        if t not in (JT["BALL"], JT["REVOLUTE"]):
            raise ValueError(f"loop joint type {t} is not supported yet")
        world = J["parent"][j] < 0
        pl = -1 if world else body_link[J["parent"][j]]
        cl = body_link[J["child"][j]]
        if cl < 0 or (not world and (pl < 0 or body_art[J["parent"][j]] != body_art[J["child"][j]])):
            raise ValueError("loop joints must close inside one articulation or to the world")
        xp, xc = J["X_p"][j], J["X_c"][j]
        ax = J["axis"][J["qd_start"][j]] if J["qd_start"][j] < len(J["axis"]) else [0, 0, 1]
        ap = quat_rotate([xp[3], xp[4], xp[5], xp[6]], ax)
        ac = quat_rotate([xc[3], xc[4], xc[5], xc[6]], ax)
        o_ = (SF["SF_LOOP"] + i * 5) * 4
        sf[o_:o_ + 20] = [pl, cl, body_art[J["child"][j]], 1 if t == JT["REVOLUTE"] else 0, xp[0], xp[1], xp[2], 0,
                          xc[0], xc[1], xc[2], 0, *ap, 0, *ac, 0]
    for i, m in enumerate(mimics):
        o_ = (SF["SF_MIMIC"] + i * 2) * 4
        sf[o_:o_ + 8] = [m["art"], m["f"], m["l"], m["c1"], m["fq"], m["lq"], m["c0"], 0]
    ctrl = S.get("control")
    ctrl_kind = ctrl_a = ctrl_b = 0
    if ctrl and ctrl.get("type") == "fader":
        ctrl_kind = 1
        ctrl_a = q_map[ctrl["fader_q"]]
        ctrl_b = dof_map[ctrl["wheel_v"]]
        sf[SF["SF_CTRL"] * 4:SF["SF_CTRL"] * 4 + 4] = [ctrl["travel"], ctrl["max_speed"], 0, 0]

    # Capacities (sim.js:395-477).
    cp = dict(MAXP=16384, MAXC=8192, MAXU=2048, UH=4096, WH=16384, MAXDENSE=512, AH=4096)
    cp.update(caps or {})
    MAXP, MAXC, MAXU, UH, WH, MAXDENSE, AH = (cp[k] for k in ("MAXP", "MAXC", "MAXU", "UH", "WH", "MAXDENSE", "AH"))
    ncolw = colorWords if colorWords is not None else o.get("colorWords", 2)
    SV = dict(body_pair_cell_size=0.06, cfm=1e-6, relaxation=1, baumgarte=0.2, contact_speculative_scale=1,
              contact_gap_gate=None, velocity_limit_activation_fraction=0, contact_friction_gap_max=None,
              contact_friction_scale=1, contact_shared_anchor=False, contact_friction_shared_anchor=False,
              contact_warmstart_decay=1, restitution_velocity_threshold=0.5, enable_restitution=True,
              contact_friction_position_iterations=-1, velocity_iterations=0, joint_limit_activation_gap=None)
    SV.update(S.get("solver") or {})
    SV.update(o.get("solver") or {})
    if o.get("warmStart") is None:
        o["warmStart"] = 1 if SV.get("contact_warmstart") else 0
    iters = o["iterations"]
    fpi = SV["contact_friction_position_iterations"]
    FMODES = ["fixed_normal", "bisection", "bisection_desaxce", "coulomb_newton"]
    fm = SV.get("friction_mode") or "fixed_normal"
    if fm not in FMODES:
        raise ValueError(f"friction_mode {fm} is not supported")
    fmode = FMODES.index(fm)
    if (SV.get("propagation_color_order") or "contact") not in ("contact", "longest_first"):
        raise ValueError(f"propagation_color_order {SV.get('propagation_color_order')} is not supported")
    for k, d in (("enable_bilateral_preelimination", False), ("propagation_same_articulation_rows", False),
                 ("update_mass_matrix_interval", 1)):
        if SV.get(k) is not None and SV[k] != d:
            raise ValueError(f"{k}={SV[k]} is not supported")
    fab = SV.get("friction_anchor_beta")
    if SV.get("enable_torsional_rolling_friction") and (fab or 0) > 0:
        raise ValueError("enable_torsional_rolling_friction needs friction_anchor_beta=0")
    anchor_beta = 0 if (fmode > 0 or SV.get("enable_torsional_rolling_friction") or SV.get("contact_compliance")) \
        else (fab if fab is not None else 0.2)
    ang_art = bool(SV.get("enable_torsional_rolling_friction"))
    fr_mut = SV.get("free_rigid_torsional_friction")
    fr_mut = -1 if fr_mut is None else fr_mut
    fr_mur = SV.get("free_rigid_rolling_friction")
    fr_mur = -1 if fr_mur is None else fr_mur
    ang_on = ang_art or fr_mut > 0 or fr_mur > 0 or any((s.get("condim") if s.get("condim") is not None else 3) >= 4
                                                      for s in S["shapes"])
    tors_on = any((s.get("torsion_radius") or 0) > 0 for s in S["shapes"])
    PO = 34 if ang_on else 19
    FMO = PO + (4 if (anchor_beta > 0 or SV.get("contact_friction_shared_anchor")) else 0)
    TO = FMO + (2 if fmode > 0 else 0)
    EO = TO + (5 if tors_on else 0)
    CO = EO + (4 if ang_art else 0)
    compliance = bool(SV.get("contact_compliance"))
    nest = bool(SV.get("nesterov_momentum"))
    MO = CO + (1 if compliance else 0)
    ROWS = MO + (2 if nest else 0)
    P = dict(P_BODY=0, P_SHAPE=NB * 2, P_AABB=NB * 2 + NS * 2, P_PREV=NB * 2 + NS * 4)
    Sd = {}
    so = 0
    for k, n in (("S_HKEY", UH), ("S_HCNT", UH), ("S_SLOT2U", UH), ("S_CSLOT", MAXC), ("S_CLOCAL", MAXC),
                 ("S_USIZE_TMP", MAXU), ("S_UKEY", MAXU), ("S_USIZE", MAXU), ("S_USTART", MAXU + 1),
                 ("S_CSTART", ncolw * 32 + 2), ("S_META", 8), ("S_CORDER", MAXC), ("S_RK0", MAXC), ("S_RK1", MAXC),
                 ("S_RK2", MAXC), ("S_KEPT", MAXC), ("S_OSTART", MAXU), ("S_LEAD", MAXC), ("S_SLOT", MAXC * 26),
                 ("S_ROWOF", MAXC), ("S_RUNIT", MAXC), ("S_PCOL", MAXC), ("S_PORD", MAXC), ("S_UTC", MAXU),
                 ("S_UTP", MAXU), ("S_UF", NB + NA), ("S_UFF", NB + NA), ("S_RCON", MAXC), ("S_WWIN", WH),
                 ("S_UWOFF", UH), ("S_WALK", MAXC), ("S_WSLOT", MAXC + MAXDENSE)):
        Sd[k] = so
        so += n
    A = {}
    ao = 0
    NQ = len(q0)
    NDA = max([1] + [a_["dofCount"] for a_ in arts])
    DHDR = 25
    DPS = DHDR + 6 * NDA
    for k, n in (("A_Q", NQ), ("A_QD", ND), ("A_QDH", ND), ("A_INT", ND), ("A_TGT", ND), ("A_TGTV", ND),
                 ("A_LIM", 2 * ND), ("A_DRV", ND), ("A_JFL", ND), ("A_JF", ND), ("A_BF", NB * 8),
                 ("A_SLP", (NB + NA) * 4), ("A_FRIC", ND), ("A_HINV", ND), ("A_LINK", max(NL, 1) * LB),
                 ("A_SNAP", NB * 8 + ND), ("A_VLG", ND + NB * 6), ("A_AVL", NA), ("A_LG", ND), ("A_RL", ND),
                 ("A_RLN", NA), ("A_ULOAD", MAXU if anchor_beta > 0 else 0), ("A_DENSE", MAXDENSE * DPS)):
        A[k] = ao
        ao += max(n, 1)
    depth = []
    for l in links:
        depth.append(depth[l["parent"]] + 1 if l["parent"] >= 0 else 1)
    C = dict(
        TGT_HELD=1 if S.get("targets_held") else 0, NEST=1 if nest else 0, MO=MO, NB=NB, NBP=max(NB, 1),
        NBP2=max(NB, 1) * 2, NCOLW=ncolw, NCOL=ncolw * 32, NS=NS, NA=NA, NAP=max(NA, 1), NL=NL, ND=ND,
        NDP=max(ND, 1), NLOOP=len(loops), NMIMIC=len(mimics), CTRL_KIND=ctrl_kind, CTRL_A=ctrl_a, CTRL_B=ctrl_b,
        NLP=max(NL, 1), NDA=NDA, JDIM=3 * NDA, MAXDENSE=MAXDENSE, DHDR=DHDR, DPS=DPS, MAXP=MAXP, MAXC=MAXC,
        MAXU=MAXU, UH=UH, WH=WH, ROWS=ROWS, PO=PO, FMO=FMO, FMODE=fmode, PATCH=1 if anchor_beta > 0 else 0,
        F_ANCHOR_BETA=anchor_beta,
        EXTRA=1 if (anchor_beta > 0 or SV.get("contact_friction_shared_anchor")) else 0,
        SHARED=1 if SV.get("contact_shared_anchor") else 0, FSHARED=1 if SV.get("contact_friction_shared_anchor") else 0,
        F_CFM=SV["cfm"], F_OMEGA=SV["relaxation"], F_SPEC=SV["contact_speculative_scale"],
        F_GAP_GATE=SV["contact_gap_gate"] if SV.get("contact_gap_gate") is not None else 1e30,
        F_FGAP=SV["contact_friction_gap_max"] if SV.get("contact_friction_gap_max") is not None else 1e30,
        F_FSCALE=SV["contact_friction_scale"], F_REST_SPEED=SV["restitution_velocity_threshold"],
        REST=1 if (SV["enable_restitution"] and not SV.get("contact_compliance")) else 0,
        PWG=1024, CSB=1024, CTI=1 if SV.get("row_schedule") == "contact_then_internal" else 0,
        SLEEP=1 if SV.get("enable_sleeping") else 0,
        F_SLEEP_LIN=SV.get("sleep_linear_threshold") if SV.get("sleep_linear_threshold") is not None else 0.05,
        F_SLEEP_ANG=SV.get("sleep_angular_threshold") if SV.get("sleep_angular_threshold") is not None else 0.15,
        F_SLEEP_TIME=SV.get("sleep_quiet_time") if SV.get("sleep_quiet_time") is not None else 0.5,
        DRIVE_ROWS=1 if SV.get("drive_mode") == "rows" else 0,
        VEL_DRIVE_ACTIVE=1 if SV.get("velocity_drive_mode") == "active" else 0,
        FUSE_VLIM=0 if SV.get("fuse_joint_velocity_limits") is False else 1,
        VLIM_ON=1 if SO.get("enable_joint_velocity_limits") else 0,
        # Not a reference option: the articulated-inertia pass's D factor/inverse and the inertia
        # accumulation into parents (up to the root) in FP64; off reproduces the reference's FP32.
        ART_F64=1 if SO.get("articulation_fp64") else 0,
        FSTART=0 if fpi < 0 else iters - min(fpi, iters), VELITERS=SV["velocity_iterations"], AH=AH,
        ANG=1 if ang_on else 0, ANG_ART=1 if ang_art else 0, F_FR_MUT=fr_mut, F_FR_MUR=fr_mur,
        JFL=1 if any(d["loadCoef"] > 0 for d in dofs) else 0, TORS=1 if tors_on else 0, TO=TO, EO=EO,
        PYRAMID=1 if SV.get("torsional_rolling_friction_cone") == "pyramidal" else 0, CO=CO,
        COMPL=1 if compliance else 0,
        F_CREEP=SV.get("torsional_rolling_friction_creep_speed") or 0, F_BP_CELL=SV["body_pair_cell_size"],
        LONGEST_FIRST=1 if SV.get("propagation_color_order") == "longest_first" else 0, SG=1, SG32=1,
        F_VLIM_FRAC=SV["velocity_limit_activation_fraction"],
        F_JL_GAP=min(SV["joint_limit_activation_gap"] if SV.get("joint_limit_activation_gap") is not None else 0.05,
                     1e30),
        F_JL_SPEED=2 if SV.get("joint_limit_activation_gap") is None else 0,
        VLIM_FREE=1 if (bodies.get("max_linear_velocity") or bodies.get("max_angular_velocity")) else 0,
        JT_REVOLUTE=JT["REVOLUTE"], JT_PRISMATIC=JT["PRISMATIC"], JT_BALL=JT["BALL"], JT_FREE=JT["FREE"],
        JT_D6=JT["D6"],
        FRICTION_COMBINE=COMBINE.index(SO.get("friction_combine") or "average"),
        RESTITUTION_COMBINE=COMBINE.index(SO.get("restitution_combine") or "average"),
        JM=6 if any(l["ndof"] > 3 for l in links) else 3,
        MAXPATH=max([1] + depth), MAXLP=max([1] + [a_["linkCount"] for a_ in arts]),
    )
    C.update(SF)
    C.update(SU)
    C.update(P)
    C.update(Sd)
    C.update(A)
    # Buffer sizes the reference allocates (sim.js:503-519), for the oracle's own allocation.
    C["LEN_STATF4"] = off
    C["LEN_STATU"] = uoff
    C["LEN_SCHED"] = so
    C["LEN_ART"] = ao

    art_init = np.zeros(ao, dtype=np.float32)
    art_init[A["A_Q"]:A["A_Q"] + NQ] = q0
    art_init[A["A_TGT"]:A["A_TGT"] + len(tq0)] = tq0
    art_init[A["A_TGTV"]:A["A_TGTV"] + len(tqd0)] = tqd0
    body_vel = np.zeros(NB * 8, dtype=np.float32)
    tw = bodies.get("twist") or []
    for b, t in enumerate(tw):
        if t is not None and body_kind[b] == 1:
            body_vel[b * 8:b * 8 + 8] = [t[0], t[1], t[2], 0, t[3], t[4], t[5], 0]
    for l in links:
        t = tw[l["body"]] if l["body"] < len(tw) else None
        if l["type"] != JT["FREE"] or l["parent"] >= 0 or not t:
            continue
        bq = bodies["q"][l["body"]]
        rc = quat_rotate([bq[3], bq[4], bq[5], bq[6]], bodies["com"][l["body"]])
        w = [t[3], t[4], t[5]]
        v = [t[0] - (w[1] * rc[2] - w[2] * rc[1]), t[1] - (w[2] * rc[0] - w[0] * rc[2]),
             t[2] - (w[0] * rc[1] - w[1] * rc[0])]
        art_init[A["A_QD"] + l["dof"]:A["A_QD"] + l["dof"] + 6] = [*v, *w]

    params = dict(
        fps=S["fps"], substeps=o["substeps"], iterations=o["iterations"], baumgarte=SV["baumgarte"],
        gravity=list(S["gravity"]), warm=o["warmStart"] * SV["contact_warmstart_decay"],
        target_frames=S.get("target_frames", 0), driven=S.get("driven", 0),
        integral_count=S.get("integral_count", 0),
        reg=0.0 if SV.get("contact_compliance") else o["regularization"])
    return Packed(C=C, statF=statF, statU=statU, body_pose=body_pose, body_vel=body_vel, art=art_init,
                  params=params, links=links, dof_map=dof_map, q_map=q_map, body_kind=list(body_kind), NB=NB, NS=NS,
                  NA=NA, NL=NL, ND=ND, NQ=NQ, joints=J, body_com=[list(c) for c in bodies["com"]],
                  layout=dict(SF=SF, SU=SU, P=P, Sd=Sd, A=A))


def substep_params(pk: Packed, substep: int, substep_count: int, phase: float, user_targets: bool = False):
    """The 112-byte ``Params`` uniform of one substep (``writeParams``, sim.js:625-639).

    Returns ``(floats[28], uints[28])`` views of the same 28 words.
    """
    p = pk.params
    buf = np.zeros(28, dtype=np.uint32)
    f = buf.view(np.float32)
    dt = 1 / p["fps"] / p["substeps"]
    f[0] = dt
    buf[1] = substep
    buf[2] = substep_count % 2
    buf[3] = p["iterations"]
    f[4] = phase
    f[5] = 1 / p["fps"]
    f[6] = p["baumgarte"]
    f[7] = 2.0
    f[8:12] = [*p["gravity"], 0]
    f[13] = p["warm"]
    buf[14] = p["target_frames"]
    buf[15] = 0 if user_targets else p["driven"]
    buf[16] = p["integral_count"]
    f[17] = p["reg"]
    return f, buf
