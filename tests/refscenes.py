"""The reference's own scene folders, packed (tests/golden/make_reference_scenes.py), and the
oracle's side of their parity runs. The oracle runs in spawned worker processes, one scene each,
so the GPU test only waits for the slowest scene."""
from __future__ import annotations

import gzip
import os
import pickle

import numpy as np

DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "_ref")
EVERY = 60       # frames between checkpoints
FRAMES = 240     # frames per scene
# Scenes whose oracle steps cheaply run 1000 frames (the metric's horizon).
LONG = {"air_hockey", "body_limits", "bounce", "box_turn", "compliance", "d6", "drives", "dumbbells", "incline",
        "kinematic", "linkages", "load_friction", "pelican_bicycle", "ragdoll", "ratio_stack", "rods", "spin_roll",
        "spinning_top", "torsion", "toy_piano", "toy_train", "toy_well", "vel_limit", "jenga", "balance_board",
        "toaster"}
LONG_FRAMES = 1020


def names() -> list[str]:
    if not os.path.isdir(DIR):
        return []
    return sorted(f[:-len(".pkl.gz")] for f in os.listdir(DIR) if f.endswith(".pkl.gz"))


def _record(name: str) -> dict:
    with gzip.open(os.path.join(DIR, name + ".pkl.gz"), "rb") as f:
        return pickle.load(f)


def load(name: str):
    """The scene packed by steel_webgpu_b200.pack (the Python restatement of Sim.build)."""
    return _record(name)["packed"]


def files(name: str) -> tuple[bytes, bytes]:
    """The scene's own files: scene.json text and scene.bin bytes."""
    r = _record(name)
    return r["json"], r["bin"]


def frames_of(name: str) -> int:
    return LONG_FRAMES if name in LONG else FRAMES


def snapshot(pk, poses, vel, art, stats):
    C = pk.C
    return dict(poses=np.array(poses[:pk.NB * 8]), vel=np.array(vel[:pk.NB * 8]),
                q=np.array(art[C["A_Q"]:C["A_Q"] + pk.NQ]), qd=np.array(art[C["A_QD"]:C["A_QD"] + pk.ND]),
                stats=np.array(stats))


def oracle_checkpoints(name: str) -> list[dict]:
    """The oracle's state every EVERY frames: poses, velocities, q, qd and the stats words
    (contacts, colors, max pairs, max units)."""
    from oracle.oracle import OracleSim
    pk = load(name)
    o = OracleSim(pk)
    out = []
    for _ in range(frames_of(name) // EVERY):
        o.step(EVERY)
        st = o.read("stats", np.uint32)
        out.append(snapshot(pk, o.read("poses"), o.read("vel"), o.read("art"), [st[5], st[6], st[4], st[3]]))
    return out
