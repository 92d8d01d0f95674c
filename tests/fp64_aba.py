"""Float64 host dynamics of a revolute articulation from its packed records, independent of the
oracle's recursive algorithm: forward kinematics from the packed joint frames, the joint-space
mass matrix H = sum_i (Jw_i^T I_i Jw_i + m_i Jv_i^T Jv_i) from each link's COM Jacobian, the
gravity forces tau = sum_i m_i Jv_i^T g plus joint springs, and the free acceleration
qdd = H^-1 tau at qd = 0 (no position/velocity drives, no applied forces). The per-dof diagonal terms
of the reference's articulated-body pass are added to H as that pass adds them to its joint-space
inertia (src/artwgsl.js:290-300): the armature and the implicit damping dt * damping. Used to
state the error of the FP32 articulated-body pass against FP64.
"""
import numpy as np


def _qmul(a, b):
    av, aw = a[:3], a[3]
    bv, bw = b[:3], b[3]
    v = aw * bv + bw * av + np.cross(av, bv)
    return np.array([v[0], v[1], v[2], aw * bw - av @ bv])


def _qrot(q, v):
    u, w = q[:3], q[3]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def _qmat(q):
    return np.stack([_qrot(q, e) for e in np.eye(3)], axis=1)


def qdd_fp64(pk, dt: float) -> np.ndarray:
    """Free joint accelerations (port dof order) of the scene's revolute links at qd = 0, for the
    substep length dt of the implicit damping term."""
    C = pk.C
    sf = pk.statF.astype(np.float64).reshape(-1, 4)
    q = pk.art[C["A_Q"]:C["A_Q"] + pk.NQ].astype(np.float64)
    g = np.array([pk.params["gravity"][k] for k in range(3)], dtype=np.float64)
    NL, ND = C["NL"], pk.ND
    lp, lq, com, jp, aw, mass, inertia = [], [], [], [], [], [], []
    dof, parent = [], []
    for l in range(NL):
        r = sf[C["SF_LINK"] + 6 * l: C["SF_LINK"] + 6 * l + 6]
        t, par, d, b = int(r[0, 0]), int(r[0, 1]), int(r[0, 2]), int(r[0, 3])
        assert t == 1, "revolute links only"
        xp_p, xp_q, xc_p, xc_q, axis = r[1, :3], r[2], r[3, :3], r[4], r[5, :3]
        qs = int(r[3, 3])
        pp, pq = (lp[par], lq[par]) if par >= 0 else (np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))
        j_p = pp + _qrot(pq, xp_p)
        j_q = _qmul(pq, xp_q)
        h = 0.5 * q[qs]
        mq = np.concatenate([axis * np.sin(h), [np.cos(h)]])
        cq = _qmul(j_q, mq)
        iq = np.array([-xc_q[0], -xc_q[1], -xc_q[2], xc_q[3]])
        l_q = _qmul(cq, iq)
        l_q /= np.linalg.norm(l_q)
        l_p = j_p + _qrot(cq, -_qrot(iq, xc_p))
        body = sf[C["SF_BODY"] + 8 * b: C["SF_BODY"] + 8 * b + 8]
        R = _qmat(l_q)
        lp.append(l_p); lq.append(l_q)
        com.append(l_p + _qrot(l_q, body[1, :3]))
        jp.append(j_p); aw.append(_qrot(j_q, axis))
        mass.append(body[1, 3]); inertia.append(R @ body[2:5, :3] @ R.T)
        dof.append(d); parent.append(par)
    H = np.zeros((ND, ND))
    tau = np.zeros(ND)
    for i in range(NL):
        Jw = np.zeros((3, ND))
        Jv = np.zeros((3, ND))
        j = i
        while j >= 0:
            Jw[:, dof[j]] = aw[j]
            Jv[:, dof[j]] = np.cross(aw[j], com[i] - jp[j])
            j = parent[j]
        H += Jw.T @ inertia[i] @ Jw + mass[i] * Jv.T @ Jv
        tau += mass[i] * Jv.T @ g
    for l in range(NL):
        rec = sf[C["SF_DOF"] + 5 * dof[l]: C["SF_DOF"] + 5 * dof[l] + 5]
        assert rec[0, 1] == 0.0 and rec[0, 2] == 0.0, "no position/velocity drives"
        H[dof[l], dof[l]] += rec[0, 0] + dt * rec[2, 0]
        qs = int(sf[C["SF_LINK"] + 6 * l + 3, 3])
        tau[dof[l]] += rec[4, 0] * (rec[4, 1] - q[qs])
    return np.linalg.solve(H, tau)
