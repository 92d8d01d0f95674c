"""Test infrastructure: ctypes harness of the CPU oracle (oracle/_build/liboracle.so).

ORACLE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
checker. The product never imports it. Parity unpinned: the reference has no golden vectors for this
path and cannot run here, so the oracle is pinned only by construction, physical known answers and
its own fixtures (tests/golden).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_LIB64 = os.path.join(_HERE, "_build", "liboracle64.so")  # all-FP64 instance (o_f64.h), the precision reference
_libs = {}


def build(quiet: bool = True) -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True, capture_output=quiet)
    return _LIB


def lib(f64: bool = False):
    """The float oracle, or with f64 its all-FP64 instance (same entry points; buffers in and out
    stay binary32 words)."""
    if f64 not in _libs:
        path = _LIB64 if f64 else _LIB
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                    ctypes.c_char_p, ctypes.c_size_t]
        for f in ("oracle_destroy", "oracle_reset", "oracle_collide"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.oracle_stage.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_sort_raw.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.oracle_set_user_targets.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_read.restype = ctypes.c_size_t
        L.oracle_read.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_write.restype = ctypes.c_int
        L.oracle_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_trig.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_atan2.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_cone5.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                                           ctypes.c_void_p]
        _libs[f64] = L
    return _libs[f64]


class OracleSim:
    """One packed scene stepped by the CPU oracle, with the reference's buffer layout. With f64 the
    all-FP64 instance steps it (every float operation in double; reads round to binary32)."""

    def __init__(self, pk, f64: bool = False):
        self.L = L = lib(f64)
        self.pk = pk
        C = pk.C
        self._keep = [np.ascontiguousarray(a) for a in (pk.statF, pk.statU, pk.body_pose, pk.body_vel, pk.art)]
        err = ctypes.create_string_buffer(256)
        self.h = L.oracle_create(pk.constants_text().encode(), self._keep[0].ctypes.data, self._keep[0].size,
                                 self._keep[1].ctypes.data, self._keep[1].size, self._keep[2].ctypes.data,
                                 self._keep[3].ctypes.data, self._keep[4].ctypes.data, self._keep[4].size, err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        self.sizes = dict(poses=(C["NB"] * 4 + C["NS"] * 4) * 4, vel=C["NB"] * 8, art=C["LEN_ART"],
                          contacts=C["MAXC"] * 6 * 4, craw=C["MAXC"] * 6 * 4, pairs=C["MAXP"] * 2,
                          sched=C["LEN_SCHED"], rows=C["MAXC"] * (C["ROWS"] + 2) * 4,
                          warm=10 * C["WH"] + 30 * C["AH"], counters=16, stats=16, collide_counts=2)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def step(self, frames=1):
        self.L.oracle_step(self.h, frames)

    def set_user_targets(self, on: bool = True):
        """Joint targets written into art[A_TGT] replace the scene's drive paths (sim.js:716-731)."""
        self.L.oracle_set_user_targets(self.h, int(on))

    def reset(self):
        self.L.oracle_reset(self.h)

    def collide(self):
        self.L.oracle_collide(self.h)

    def sort_raw(self, n: int):
        """The canonical contact sort alone over the first n raw records (after write("craw"))."""
        self.L.oracle_sort_raw(self.h, n)

    def stage(self, k: int):
        self.L.oracle_stage(self.h, k)

    def read(self, name, dtype=np.float32):
        n = self.sizes[name]
        out = np.zeros(n, dtype=np.uint32)
        got = self.L.oracle_read(self.h, name.encode(), out.ctypes.data, n)
        return out[:got].view(dtype)

    def write(self, name, offset, values, dtype=np.float32):
        a = np.ascontiguousarray(np.asarray(values, dtype=dtype))
        if self.L.oracle_write(self.h, name.encode(), offset, a.ctypes.data, a.size) != 0:
            raise IndexError(name)

    def body_poses(self):
        """(NB, 8): COM position, 0, quaternion."""
        nb = self.pk.NB
        return self.read("poses")[:nb * 8].reshape(nb, 8)


def trig(x):
    """The oracle's float sin and cos of x (float32 array)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    s, c = np.zeros_like(x), np.zeros_like(x)
    lib().oracle_trig(x.ctypes.data, s.ctypes.data, c.ctypes.data, x.size)
    return s, c


def atan2(y, x):
    """The oracle's float atan2(y, x)."""
    y = np.ascontiguousarray(y, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros_like(y)
    lib().oracle_atan2(y.ctypes.data, x.ctypes.data, out.ctypes.data, y.size)
    return out


def cone5(H, g, mu, lam, load, pyramidal=False, creep=0.0, omega=1.0):
    """The oracle's articulated angular friction block (t1, t2, spin, roll1, roll2): new impulses."""
    a = [np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1)) for x in (H, g, mu, lam)]
    out = np.zeros(5, dtype=np.float32)
    lib().oracle_cone5(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, a[3].ctypes.data, load, int(pyramidal),
                       creep, omega, out.ctypes.data)
    return out
