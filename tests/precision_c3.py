"""Precision report of the articulation workload: PD-driven quadrupeds plus 40-link chains with
link mass ratios log-uniform 1-1e3, 500 fps, 4 substeps, 12 iterations.

Test infrastructure (runs the CPU oracle only). Three runs of the same scene and the same target
sequence:
- "fp32": the float path (bit-identical to the CUDA path, as the GPU parity tests show);
- "fp32+fp64 D^-1": the float path with the FP64 branch of the articulated-inertia pass (the
  joint-space D = S^T I^A S factor and inverse and the root spatial-inertia accumulation,
  artwgsl.js:192-207 and :342), bit-identical to the CUDA path's `articulation_fp64` instance;
- "fp64": the oracle's all-FP64 instance (o_f64.h), the precision reference.
The chains start from joint angles uniform in +-0.5 rad, so that they swing. PD targets are
uniform in +-0.5 rad and resampled every 50 frames (seeded), written as the
reference's setJointTargets writes them (sim.js:716-731). At checkpoint frames the report gives,
for the quadrupeds' bodies and the chains' bodies apart, the relative L2 error against the FP64 run
(||x - x64|| / ||x64||) of COM positions, orientations (quaternion difference with the sign fixed),
linear and angular velocities, joint coordinates q and joint velocities qd.

    python tests/precision_c3.py                      # 1024 quadrupeds + 64 chains, 1000 frames
    python tests/precision_c3.py --quads 16 --chains 2 --frames 200
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

QUAD_BODIES = 13  # floating base + 4 legs of 3 links
LEGS = ("fp32", "fp32+fp64 D^-1", "fp64")
QUANTITIES = ("position", "orientation", "linear velocity", "angular velocity", "q", "qd")


def build(quads: int, chains: int, links: int, seed: int, swing: float):
    """The scene packed twice (float, and with the FP64 D^-1 branch), the PD joints' Newton dofs.
    The chains start from joint angles uniform in +-swing rad (they hang at rest otherwise)."""
    from steel_webgpu_b200 import synth
    from steel_webgpu_b200.packer import pack
    from steel_webgpu_b200.sim import auto_caps
    sc = synth.quadrupeds(quads, chains, links, seed=seed)
    caps = auto_caps(sc)
    pd = [int(d) for d in sc.json["info"]["pd_joints"]]
    pks = [pack(sc, caps=caps), pack(sc, opts={"solver": {"articulation_fp64": True}}, caps=caps)]
    chain_q = [pks[0].q_map[n] for n in range(quads * (7 + 12), quads * (7 + 12) + chains * links)]
    angles = np.random.default_rng(seed + 1).uniform(-swing, swing, len(chain_q)).astype(np.float32)
    for pk in pks:
        pk.art[[pk.C["A_Q"] + q for q in chain_q]] = angles
    return pks[0], pks[1], pd


def snapshot(o, pk):
    """Body COM positions and quaternions, body twists (articulated bodies from their link record),
    q and qd, all as float64 arrays."""
    from steel_webgpu_b200.packer import LB, L_V
    C = pk.C
    nb = pk.NB
    poses = o.read("poses")[:nb * 8].reshape(nb, 8).astype(np.float64)
    vel = o.read("vel")[:nb * 8].reshape(nb, 8).astype(np.float64)
    art = o.read("art").astype(np.float64)
    for l, link in enumerate(pk.links):
        r = C["A_LINK"] + l * LB + L_V
        vel[link["body"], 0:3] = art[r + 3:r + 6]
        vel[link["body"], 4:7] = art[r:r + 3]
    return dict(pos=poses[:, 0:3], quat=poses[:, 4:8], lin=vel[:, 0:3], ang=vel[:, 4:7],
                q=art[C["A_Q"]:C["A_Q"] + pk.NQ], qd=art[C["A_QD"]:C["A_QD"] + pk.ND])


def run_leg(args):
    """One run: steps the scene, resampling targets every 50 frames, and returns its snapshots at
    the checkpoint frames."""
    leg, pk, pd, frames, checkpoints, seed = args
    from oracle.oracle import OracleSim
    o = OracleSim(pk, f64=(leg == "fp64"))
    rng = np.random.default_rng(seed)
    A_TGT = pk.C["A_TGT"]
    port = [pk.dof_map[d] for d in pd]
    out = {}
    blowup = None  # first frame after which a body pose is not finite
    nb = pk.NB
    t0 = time.time()
    for f in range(frames):
        if f % 50 == 0:
            tg = rng.uniform(-0.5, 0.5, len(port)).astype(np.float32)
            for d, v in zip(port, tg):
                o.write("art", A_TGT + d, [v])
            o.set_user_targets(True)
        o.step(1)
        if blowup is None and not np.isfinite(o.read("poses")[:nb * 8]).all():
            blowup = f + 1
        if f + 1 in checkpoints:
            out[f + 1] = snapshot(o, pk)
    out["blowup"] = blowup
    return leg, out, time.time() - t0


def rel(a, r):
    d = np.linalg.norm(r)
    return float(np.linalg.norm(a - r) / d) if d > 0 else float(np.linalg.norm(a - r))


def groups(pk, quads: int):
    """Bodies, port coordinates and port dofs of the quadrupeds and of the chains (the quadrupeds
    come first in Newton order: 13 bodies, 19 coordinates and 18 dofs each)."""
    qn, dn = quads * 19, quads * 18
    quad_q = np.array(sorted(p for n, p in pk.q_map.items() if n < qn), dtype=np.int64)
    chain_q = np.array(sorted(p for n, p in pk.q_map.items() if n >= qn), dtype=np.int64)
    quad_d = np.array(sorted(p for n, p in pk.dof_map.items() if n < dn), dtype=np.int64)
    chain_d = np.array(sorted(p for n, p in pk.dof_map.items() if n >= dn), dtype=np.int64)
    nb = quads * QUAD_BODIES
    return {"quadrupeds": (slice(0, nb), quad_q, quad_d), "chains": (slice(nb, None), chain_q, chain_d)}


def errors(s, ref, grp):
    """Relative L2 error per quantity, for the quadrupeds and the chains apart."""
    out = {}
    for group, (sl, qi, di) in grp.items():
        if s["pos"][sl].size == 0:
            continue
        qa, qr = s["quat"][sl], ref["quat"][sl]
        sign = np.where(np.sum(qa * qr, axis=1, keepdims=True) < 0, -1.0, 1.0)
        out[group] = {"position": rel(s["pos"][sl], ref["pos"][sl]), "orientation": rel(qa * sign, qr),
                      "linear velocity": rel(s["lin"][sl], ref["lin"][sl]),
                      "angular velocity": rel(s["ang"][sl], ref["ang"][sl]),
                      "q": rel(s["q"][qi], ref["q"][qi]), "qd": rel(s["qd"][di], ref["qd"][di])}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--quads", type=int, default=1024)
    ap.add_argument("--chains", type=int, default=64)
    ap.add_argument("--links", type=int, default=40)
    ap.add_argument("--frames", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--swing", type=float, default=0.5, help="chains' initial joint angles, uniform in +-swing rad")
    ap.add_argument("--out", default=None, help="write the report as JSON here")
    a = ap.parse_args(argv)
    checkpoints = sorted({c for c in (1, 10, 50, 100, 200, 500, 1000, a.frames) if c <= a.frames})
    t0 = time.time()
    pk32, pk64d, pd = build(a.quads, a.chains, a.links, a.seed, a.swing)
    print(f"scene: {a.quads} quadrupeds + {a.chains} x {a.links}-link chains, {pk32.NB} bodies, {pk32.ND} dofs; "
          f"built in {time.time() - t0:.0f} s", flush=True)
    jobs = [("fp32", pk32, pd, a.frames, checkpoints, a.seed), ("fp32+fp64 D^-1", pk64d, pd, a.frames, checkpoints, a.seed),
            ("fp64", pk32, pd, a.frames, checkpoints, a.seed)]
    with mp.get_context("spawn").Pool(3) as pool:
        res = {leg: (snaps, secs) for leg, snaps, secs in pool.map(run_leg, jobs)}
    ref = res["fp64"][0]
    report = {"scene": dict(quads=a.quads, chains=a.chains, links=a.links, bodies=pk32.NB, dofs=pk32.ND, fps=500,
                            frames=a.frames, seed=a.seed, swing=a.swing),
              "seconds": {leg: round(res[leg][1], 1) for leg in LEGS},
              "first_nonfinite_frame": {leg: res[leg][0].pop("blowup") for leg in LEGS}, "errors": {}}
    grp = groups(pk32, a.quads)
    for leg in LEGS[:2]:
        report["errors"][leg] = {f: errors(res[leg][0][f], ref[f], grp) for f in checkpoints}
    print("first frame with a non-finite body pose (None: finite throughout):", report["first_nonfinite_frame"])
    print("relative L2 error against the all-FP64 run")
    print(f"{'frame':>6} {'run':<16} {'group':<11} " + " ".join(f"{q:>16}" for q in QUANTITIES))
    for f in checkpoints:
        for leg in LEGS[:2]:
            e = report["errors"][leg][f]
            for group in ("quadrupeds", "chains"):
                if group not in e:
                    continue
                vals = [e[group][q] for q in QUANTITIES]
                print(f"{f:>6} {leg:<16} {group:<11} " + " ".join(f"{v:16.3e}" for v in vals))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(report, fh, indent=1)
    return report


if __name__ == "__main__":
    main()
