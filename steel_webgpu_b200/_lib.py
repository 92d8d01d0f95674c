"""ctypes binding of libsteel_b200.so (include/steel_b200.h).

The library is built in-tree (``steel_webgpu_b200/build.py``). There is no CPU fallback: loading
fails loudly when the shared library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsteel_b200.so")

STEEL_OK = 0
ERRORS = {1: "invalid", 2: "unsupported", 3: "capacity", 4: "cuda", 5: "nomem", 6: "nodevice", 7: "timeout"}


class SteelError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"steel error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class SceneDesc(ctypes.Structure):
    _fields_ = [("constants", ctypes.c_char_p), ("statF", ctypes.c_void_p), ("statF_floats", ctypes.c_uint64),
                ("statU", ctypes.c_void_p), ("statU_words", ctypes.c_uint64), ("body_pose", ctypes.c_void_p),
                ("body_vel", ctypes.c_void_p), ("art", ctypes.c_void_p), ("art_floats", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("max_contacts", "max_colors", "max_units", "max_pairs", "contacts",
                                               "colors", "max_dense", "asleep", "overflow")]


class Tiles(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("block_threads", "smem_budget", "narrow_blocks_per_sm", "stream_groups")]


class NewtonInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("bodies", "joint_coords", "joint_dofs")]


class SceneInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("NB", "NS", "NA", "NL", "ND", "NQ", "max_pairs", "max_contacts",
                                               "max_units", "max_dense")]


# Every entry point the header declares, with its argument types.
_VP = ctypes.c_void_p
_U32 = ctypes.c_uint32
_F32 = ctypes.c_float
_FP = ctypes.POINTER(ctypes.c_float)
SIGNATURES = {
    "steel_ctx_create": [ctypes.c_int, ctypes.POINTER(_VP)],
    "steel_ctx_destroy": [_VP],
    "steel_last_error": [],
    "steel_batch_create": [_VP, ctypes.POINTER(SceneDesc), _U32, ctypes.POINTER(_VP)],
    "steel_batch_destroy": [_VP],
    "steel_scene_create": [_VP, ctypes.c_char_p, ctypes.c_uint64, _VP, ctypes.c_uint64, ctypes.c_char_p,
                           ctypes.POINTER(_VP)],
    "steel_batch_create_files": [_VP, _U32, _VP, _VP, _VP, _VP, _VP, ctypes.POINTER(_VP)],
    "steel_convex_hull": [_VP, _U32, _VP, _VP, _VP, _VP, ctypes.POINTER(_U32), ctypes.POINTER(_U32)],
    "steel_pack": [ctypes.c_char_p, ctypes.c_uint64, _VP, ctypes.c_uint64, ctypes.c_char_p, ctypes.POINTER(_VP)],
    "steel_packed_desc": [_VP, ctypes.POINTER(SceneDesc)],
    "steel_packed_free": [_VP],
    "steel_newton_info": [_VP, _U32, ctypes.POINTER(NewtonInfo)],
    "steel_state": [_VP, _U32, _VP, _VP, _VP, _VP],
    "steel_newton_dof": [_VP, _U32, _U32, ctypes.POINTER(_U32)],
    "steel_scene_info_get": [_VP, _U32, ctypes.POINTER(SceneInfo)],
    "steel_reset": [_VP],
    "steel_step": [_VP, _U32],
    "steel_sync": [_VP],
    "steel_set_graph": [_VP, ctypes.c_int],
    "steel_get_tiles": [_VP, ctypes.POINTER(Tiles)],
    "steel_set_tiles": [_VP, ctypes.POINTER(Tiles)],
    "steel_autotune": [_VP, _U32, ctypes.POINTER(Tiles), ctypes.POINTER(_F32)],
    "steel_set_team": [_VP, _U32],
    "steel_get_team": [_VP, ctypes.POINTER(_U32)],
    "steel_read_poses": [_VP, _U32, _VP],
    "steel_read_state": [_VP, _U32, _VP, _VP, _VP, _VP, _VP],
    "steel_copy_poses_device": [_VP, _U32, _VP, _VP],
    "steel_get_stats": [_VP, _U32, ctypes.POINTER(Stats)],
    "steel_set_joint_target": [_VP, _U32, _U32, _F32, _F32],
    "steel_set_joint_force": [_VP, _U32, _U32, _F32],
    "steel_set_body_wrench": [_VP, _U32, _U32, _FP, _FP],
    "steel_set_body_pose": [_VP, _U32, _U32, _FP, _FP],
    "steel_set_body_twist": [_VP, _U32, _U32, _FP],
    "steel_collide": [_VP],
    "steel_read_pairs": [_VP, _U32, _VP, _U32, ctypes.POINTER(_U32)],
    "steel_read_contacts": [_VP, _U32, _VP, _U32, ctypes.POINTER(_U32)],
    "steel_debug_stage": [_VP, ctypes.c_int],
    "steel_read_words": [_VP, _U32, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, _VP],
    "steel_layout_get": [_VP, _U32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)],
    "steel_step_timed": [_VP, _U32, ctypes.POINTER(_F32)],
    "steel_debug_set_wait_limit": [_VP, _U32],
    "steel_step_io": [_VP, _U32, _VP, ctypes.c_uint64, _VP, ctypes.c_uint64],
    "steel_profile_kernels": [_VP, _U32, _VP],
    "steel_trace": [_VP, ctypes.c_int],
    "steel_trace_read": [_VP, _VP, ctypes.c_uint64],
    "steel_sort_contacts_noalloc": [_VP, _U32, _VP, _VP],
    "steel_serve_config": [_VP, _U32],
    "steel_serve_budget": [_VP, ctypes.c_uint64],
    "steel_scene_bytes": [_VP, _U32, ctypes.POINTER(ctypes.c_uint64)],
    "steel_serve_submit": [_VP, _U32, _U32, ctypes.POINTER(ctypes.c_uint64)],
    "steel_serve_tick": [_VP, ctypes.POINTER(_U32)],
    "steel_serve_poll": [_VP, _VP, _VP, _VP, _U32, ctypes.POINTER(_U32)],
    "steel_serve_end": [_VP],
}

_lib = None


def load(path: str = LIB_PATH):
    """Loads the library (no GPU needed to load; calls that launch work need one)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m steel_webgpu_b200.build`")
    L = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_char_p if name == "steel_last_error" else ctypes.c_int
    _lib = L
    return L


def check(rc: int):
    if rc != STEEL_OK:
        raise SteelError(rc, load().steel_last_error().decode())
