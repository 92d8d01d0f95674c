"""The reference's ``Sim`` API over the CUDA library.

Mirrors ``packages/steel-webgpu/src/sim.js`` (class ``Sim``, typed in ``src/sim.d.ts:53-92``):
construction packs the scene (``packer.pack``, the restatement of ``Sim.build``) and hands the
packed buffers to the C ABI; ``step``/``reset``/``state``/``poses``/``stats`` and the setters keep
their names, argument meaning and errors. ``Batch`` steps many scenes in one launch sequence.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .builder import JT, LoadedScene
from .packer import LB, L_V, Packed, pack, quat_rotate


def auto_caps(scene: LoadedScene) -> dict:
    """Capacities sized to a scene instead of the reference's fixed MAXP/MAXC (sim.js:396).

    Results depend on capacities only when one overflows; the hash tables (WH, AH) only need room.
    """
    ns = sum(1 for s in scene.json["shapes"] if s.get("hull") or s.get("plane"))
    # Piles of the uneven batch peak near 4 pairs and 2.5 contacts per shape; these leave 2-5x room.
    maxp = int(min(max(256, 8 * ns), 1 << 22))
    maxc = int(min(max(512, 12 * ns), 1 << 24))
    # Same-articulation contacts: a 40-link chain keeps about 3 per link (links two apart touch).
    maxdense = int(min(max(512, 4 * int(scene.json["joints"].get("count", 0))), 1 << 20))

    def p2(x):
        return 1 << max(int(x) - 1, 1).bit_length()

    return dict(MAXP=maxp, MAXC=maxc, MAXU=maxc, UH=p2(maxc), WH=p2(2 * maxc), AH=p2(maxc), MAXDENSE=maxdense)


class _Context:
    _by_device: dict = {}

    @classmethod
    def get(cls, device: int):
        h = cls._by_device.get(device)
        if h is None:
            L = _lib.load()
            p = ctypes.c_void_p()
            _lib.check(L.steel_ctx_create(device, ctypes.byref(p)))
            h = p.value
            cls._by_device[device] = h
        return h


class Batch:
    """Packed scenes stepped together on one GPU (one batch = one launch sequence per substep)."""

    def __init__(self, packed: list[Packed], device: int = 0, graph: bool = True):
        L = _lib.load()
        self.packed = list(packed)
        self._keep = []
        descs = (_lib.SceneDesc * len(self.packed))()
        for i, pk in enumerate(self.packed):
            arrs = [np.ascontiguousarray(a) for a in (pk.statF, pk.statU, pk.body_pose, pk.body_vel, pk.art)]
            text = pk.constants_text().encode()
            self._keep.append((arrs, text))
            descs[i] = _lib.SceneDesc(text, arrs[0].ctypes.data, arrs[0].size, arrs[1].ctypes.data, arrs[1].size,
                                      arrs[2].ctypes.data, arrs[3].ctypes.data, arrs[4].ctypes.data, arrs[4].size)
        ctx = _Context.get(device)
        h = ctypes.c_void_p()
        _lib.check(L.steel_batch_create(ctx, descs, len(self.packed), ctypes.byref(h)))
        self.h = h.value
        self.n_scenes = len(self.packed)
        self._keep.clear()
        if not graph:
            _lib.check(L.steel_set_graph(self.h, 0))

    @classmethod
    def from_files(cls, scenes: list, device: int = 0, graph: bool = True) -> "Batch":
        """A batch created from the scenes' own files through the C ABI (steel_batch_create_files: the
        library reads scene.json and packs in C++). scenes: (json text bytes, bin bytes, options dict or
        None) per scene."""
        import json as _json
        L = _lib.load()
        n = len(scenes)
        texts = [t if isinstance(t, bytes) else t.encode() for t, _, _ in scenes]
        bins = [ctypes.create_string_buffer(bytes(b), len(b)) for _, b, _ in scenes]
        opts = [(_json.dumps(o).encode() if o else None) for _, _, o in scenes]
        jp = (ctypes.c_char_p * n)(*texts)
        jl = (ctypes.c_uint64 * n)(*[len(t) for t in texts])
        bp = (ctypes.c_void_p * n)(*[ctypes.cast(b, ctypes.c_void_p) for b in bins])
        bl = (ctypes.c_uint64 * n)(*[len(sc[1]) for sc in scenes])
        op = (ctypes.c_char_p * n)(*opts)
        h = ctypes.c_void_p()
        _lib.check(L.steel_batch_create_files(_Context.get(device), n, jp, jl, bp, bl, op, ctypes.byref(h)))
        self = cls.__new__(cls)
        self.packed = []
        self._keep = []
        self.h = h.value
        self.n_scenes = n
        if not graph:
            _lib.check(L.steel_set_graph(self.h, 0))
        return self

    def close(self):
        if getattr(self, "h", None):
            _lib.load().steel_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, frames: int = 1):
        _lib.check(_lib.load().steel_step(self.h, frames))

    def step_timed(self, frames: int = 1) -> float:
        ms = ctypes.c_float()
        _lib.check(_lib.load().steel_step_timed(self.h, frames, ctypes.byref(ms)))
        return ms.value

    def sync(self):
        _lib.check(_lib.load().steel_sync(self.h))

    def step_io(self, frames: int, targets: np.ndarray | None, poses_out: np.ndarray | None):
        """One control step through host memory: packed joint targets in, packed body poses out."""
        t = targets.ctypes.data if targets is not None else None
        nt = targets.size if targets is not None else 0
        p = poses_out.ctypes.data if poses_out is not None else None
        npz = poses_out.size if poses_out is not None else 0
        _lib.check(_lib.load().steel_step_io(self.h, frames, t, nt, p, npz))

    def profile_kernels(self, frames: int) -> dict:
        out = np.zeros(7, dtype=np.float32)
        _lib.check(_lib.load().steel_profile_kernels(self.h, frames, out.ctypes.data))
        return dict(zip(["params", "shapes", "broad", "narrow", "csort", "prepare", "solve"], out.tolist()))

    def reset(self):
        _lib.check(_lib.load().steel_reset(self.h))

    def trace(self, on: bool = True):
        """Turns the per-scene block trace of the prepare and solve kernels on or off."""
        _lib.check(_lib.load().steel_trace(self.h, 1 if on else 0))

    def trace_read(self) -> dict:
        """The last prepare and solve launches' block records, per scene: start and end (global
        timer, ns) and SM, as int64 arrays of shape (n_scenes, 3)."""
        n = self.n_scenes
        out = np.zeros(6 * n, dtype=np.uint64)
        _lib.check(_lib.load().steel_trace_read(self.h, out.ctypes.data, out.size))
        rec = out.astype(np.int64).reshape(2, n, 3)
        return {"prepare": rec[0], "solve": rec[1]}

    def tiles(self) -> dict:
        t = _lib.Tiles()
        _lib.check(_lib.load().steel_get_tiles(self.h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _lib.Tiles._fields_}

    def set_tiles(self, block_threads: int, smem_budget: int = 0, narrow_blocks_per_sm: int = 0, stream_groups: int = 1):
        t = _lib.Tiles(block_threads, smem_budget, narrow_blocks_per_sm, stream_groups)
        _lib.check(_lib.load().steel_set_tiles(self.h, ctypes.byref(t)))

    TEAM_AUTO = 0xFFFFFFFF

    def set_team(self, blocks: int = TEAM_AUTO):
        """Blocks that solve the batch's one scene together (steel_set_team): 0 one block,
        TEAM_AUTO the default rule for large scenes, else that many."""
        _lib.check(_lib.load().steel_set_team(self.h, blocks))

    def team(self) -> int:
        """Blocks of the team solve in use (0: one block per scene)."""
        v = ctypes.c_uint32()
        _lib.check(_lib.load().steel_get_team(self.h, ctypes.byref(v)))
        return v.value

    def autotune(self, frames: int = 3) -> tuple[dict, float]:
        """Times each candidate tile configuration over `frames` frames from the initial state, keeps
        the fastest and resets the batch. Returns (tiles, ms per frame)."""
        t = _lib.Tiles()
        ms = ctypes.c_float()
        _lib.check(_lib.load().steel_autotune(self.h, frames, ctypes.byref(t), ctypes.byref(ms)))
        return {k: getattr(t, k) for k, _ in _lib.Tiles._fields_}, ms.value

    def scene_bytes(self, scene: int = 0) -> int:
        """Bytes of the scene's state in the batch arena (the serving budget's unit)."""
        v = ctypes.c_uint64()
        _lib.check(_lib.load().steel_scene_bytes(self.h, scene, ctypes.byref(v)))
        return v.value

    def info(self, scene: int = 0) -> _lib.SceneInfo:
        out = _lib.SceneInfo()
        _lib.check(_lib.load().steel_scene_info_get(self.h, scene, ctypes.byref(out)))
        return out

    def poses(self, scene: int = 0) -> np.ndarray:
        nb = self.packed[scene].NB
        out = np.zeros(nb * 8, dtype=np.float32)
        _lib.check(_lib.load().steel_read_poses(self.h, scene, out.ctypes.data))
        return out

    def raw_state(self, scene: int = 0):
        pk = self.packed[scene]
        poses = np.zeros(pk.NB * 8, dtype=np.float32)
        vel = np.zeros(pk.NB * 8, dtype=np.float32)
        q = np.zeros(max(pk.NQ, 1), dtype=np.float32)
        qd = np.zeros(max(pk.ND, 1), dtype=np.float32)
        lv = np.zeros(max(pk.NL, 1) * 6, dtype=np.float32)
        _lib.check(_lib.load().steel_read_state(self.h, scene, poses.ctypes.data, vel.ctypes.data, q.ctypes.data,
                                                qd.ctypes.data, lv.ctypes.data))
        return poses, vel, q[:pk.NQ], qd[:pk.ND], lv[:pk.NL * 6]

    def stats(self, scene: int = 0) -> dict:
        s = _lib.Stats()
        _lib.check(_lib.load().steel_get_stats(self.h, scene, ctypes.byref(s)))
        out = {k: getattr(s, k) for k, _ in _lib.Stats._fields_ if k != "overflow"}
        names = ["pairs", "contacts", "units", "dense rows"]
        out["overflow"] = [n for i, n in enumerate(names) if s.overflow & (1 << i)]
        return out

    def debug_stage(self, stage: int):
        _lib.check(_lib.load().steel_debug_stage(self.h, stage))

    def layout(self, key: str, scene: int = 0) -> int:
        v = ctypes.c_uint64()
        _lib.check(_lib.load().steel_layout_get(self.h, scene, key.encode(), ctypes.byref(v)))
        return v.value

    def read_words(self, buffer: str, offset: int, count: int, scene: int = 0, dtype=np.float32) -> np.ndarray:
        out = np.zeros(max(count, 1), dtype=np.uint32)
        _lib.check(_lib.load().steel_read_words(self.h, scene, buffer.encode(), offset, count, out.ctypes.data))
        return out[:count].view(dtype)

    def collide(self):
        _lib.check(_lib.load().steel_collide(self.h))

    def pairs(self, scene: int = 0) -> np.ndarray:
        L = _lib.load()
        n = ctypes.c_uint32()
        _lib.check(L.steel_read_pairs(self.h, scene, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1) * 2, dtype=np.uint32)
        _lib.check(L.steel_read_pairs(self.h, scene, out.ctypes.data, n.value, ctypes.byref(n)))
        return out[:n.value * 2].reshape(-1, 2)

    def contacts(self, scene: int = 0):
        """Sorted contact records (nc, 5, 4) and shape-mu pairs (nc, 4)."""
        L = _lib.load()
        n = ctypes.c_uint32()
        _lib.check(L.steel_read_contacts(self.h, scene, None, 0, ctypes.byref(n)))
        nc = n.value
        out = np.zeros(max(nc, 1) * 24, dtype=np.float32)
        _lib.check(L.steel_read_contacts(self.h, scene, out.ctypes.data, nc, ctypes.byref(n)))
        return out[:nc * 20].reshape(nc, 5, 4), out[nc * 20:nc * 24].reshape(nc, 4)


class Server:
    """Continuous batching over a Batch's scenes as resident instances (steel_serve_*).

    ``submit(instance, frames)`` queues a request; ``tick()`` steps every admitted instance by one
    frame; ``poll()`` returns finished requests with their latency (submit to completion, ms).
    """

    def __init__(self, batch: Batch, max_active: int = 0, budget_bytes: int = 0):
        self.batch = batch
        _lib.check(_lib.load().steel_serve_config(batch.h, max_active))
        _lib.check(_lib.load().steel_serve_budget(batch.h, budget_bytes))

    def submit(self, instance: int, frames: int) -> int:
        rid = ctypes.c_uint64()
        _lib.check(_lib.load().steel_serve_submit(self.batch.h, instance, frames, ctypes.byref(rid)))
        return rid.value

    def tick(self) -> int:
        n = ctypes.c_uint32()
        _lib.check(_lib.load().steel_serve_tick(self.batch.h, ctypes.byref(n)))
        return n.value

    def poll(self, cap: int = 4096) -> list:
        ids = np.zeros(cap, dtype=np.uint64)
        inst = np.zeros(cap, dtype=np.uint32)
        lat = np.zeros(cap, dtype=np.float64)
        n = ctypes.c_uint32()
        _lib.check(_lib.load().steel_serve_poll(self.batch.h, ids.ctypes.data, inst.ctypes.data, lat.ctypes.data,
                                                cap, ctypes.byref(n)))
        return [(int(ids[k]), int(inst[k]), float(lat[k])) for k in range(n.value)]

    def close(self):
        _lib.check(_lib.load().steel_serve_end(self.batch.h))


class Sim:
    """``new Sim(device, scene, opts)`` (sim.js:63-75) as a batch of one scene."""

    def __init__(self, scene: LoadedScene, opts: dict | None = None, device: int = 0, caps: dict | str | None = None,
                 graph: bool = True):
        if caps == "auto":
            caps = auto_caps(scene)
        self.scene = scene
        self.packed = pack(scene, opts, caps=caps)
        self.C = self.packed.C
        self.NB = self.packed.NB
        self.bodyKind = self.packed.body_kind
        self.time = 0.0
        self.frame = 0
        self._batch = Batch([self.packed], device=device, graph=graph)

    # --- lifecycle (sim.js:85-93, 613-623) ---
    def destroy(self):
        self._batch.close()

    def reset(self):
        self._batch.reset()
        self.time = 0.0
        self.frame = 0

    # --- stepping (sim.js:692-712) ---
    def step(self, frames: int = 1):
        self._batch.step(frames)
        self.frame += frames
        self.time += frames / self.scene.json["fps"]

    def run(self, frames: int, on_frame=None):
        for _ in range(frames):
            if on_frame is not None:
                on_frame(self, self.frame)
            self.step(1)
        self._batch.sync()

    # --- readback (sim.js:732-763, 804, 822-834) ---
    def poses(self) -> np.ndarray:
        return self._batch.poses()

    def state(self) -> dict:
        pk = self.packed
        J = pk.joints
        poses, vel, q, qd, lv = self._batch.raw_state()
        vel = vel.copy()
        for l, link in enumerate(pk.links):
            b = link["body"]
            o = l * 6
            vel[b * 8:b * 8 + 8] = [lv[o + 3], lv[o + 4], lv[o + 5], 0, lv[o], lv[o + 1], lv[o + 2], 0]
        NB = pk.NB
        bodyQ = np.zeros(NB * 7, dtype=np.float32)
        bodyQd = np.zeros(NB * 6, dtype=np.float32)
        for b in range(NB):
            qv = poses[b * 8 + 4:b * 8 + 8].astype(np.float64)
            r = quat_rotate(qv, pk.body_com[b])
            bodyQ[b * 7:b * 7 + 7] = [poses[b * 8] - r[0], poses[b * 8 + 1] - r[1], poses[b * 8 + 2] - r[2], *qv]
            bodyQd[b * 6:b * 6 + 6] = [vel[b * 8], vel[b * 8 + 1], vel[b * 8 + 2], vel[b * 8 + 4], vel[b * 8 + 5],
                                       vel[b * 8 + 6]]
        jointQ = np.asarray(J["q"], dtype=np.float32).copy()
        jointQd = np.zeros(J["qd_start"][-1], dtype=np.float32)
        for nq, qi in pk.q_map.items():
            jointQ[nq] = q[qi]
        for nd, di in pk.dof_map.items():
            jointQd[nd] = qd[di]
        for j, t in enumerate(J["type"]):
            if t not in (JT["FREE"], JT["DISTANCE"]) or J["q_start"][j] in pk.q_map:
                continue
            b = J["child"][j]
            jointQ[J["q_start"][j]:J["q_start"][j] + 7] = bodyQ[b * 7:b * 7 + 7]
            jointQd[J["qd_start"][j]:J["qd_start"][j] + 6] = bodyQd[b * 6:b * 6 + 6]
        return dict(bodyQ=bodyQ, bodyQd=bodyQd, jointQ=jointQ, jointQd=jointQd)

    def stats(self) -> dict:
        return self._batch.stats()

    # --- user control (sim.js:716-785) ---
    def setJointTarget(self, newtonDof: int, pos: float, vel: float = 0.0):
        d = self.packed.dof_map.get(newtonDof)
        if d is None:
            raise ValueError(f"dof {newtonDof} is not simulated as an articulation dof")
        _lib.check(_lib.load().steel_set_joint_target(self._batch.h, 0, d, pos, vel))

    def setJointTargets(self, pos, vel=None, first: int = 0):
        for k in range(len(pos)):
            self.setJointTarget(first + k, float(pos[k]), float(vel[k]) if vel is not None else 0.0)

    def setJointForce(self, newtonDof: int, value: float):
        d = self.packed.dof_map.get(newtonDof)
        if d is None:
            raise ValueError(f"dof {newtonDof} is not simulated as an articulation dof")
        _lib.check(_lib.load().steel_set_joint_force(self._batch.h, 0, d, value))

    def setBodyWrench(self, body: int, force, torque):
        f = (ctypes.c_float * 3)(*force)
        t = (ctypes.c_float * 3)(*torque)
        _lib.check(_lib.load().steel_set_body_wrench(self._batch.h, 0, body, f, t))

    def setBodyPose(self, body: int, com, quat):
        c = (ctypes.c_float * 3)(*com)
        q = (ctypes.c_float * 4)(*quat)
        _lib.check(_lib.load().steel_set_body_pose(self._batch.h, 0, body, c, q))

    def setBodyTwist(self, body: int, twist):
        t = (ctypes.c_float * 6)(*twist)
        _lib.check(_lib.load().steel_set_body_twist(self._batch.h, 0, body, t))
