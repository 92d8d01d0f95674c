"""Packs the reference's own scene folders (``assets/scenes/*/scene.json`` + ``scene.bin`` of
skild-ai/steel-webgpu) into test fixtures for the CUDA-vs-oracle parity test
(tests/test_reference_scenes_gpu.py).

The folders only exist where the reference is checked out, and the GPU box has no copy, so this
script packs each scene with ``steel_webgpu_b200.pack`` (the restatement of sim.js:95-521) and
writes the packed scene (a pickled ``Packed``) with the scene.json text and scene.bin bytes it came
from to ``tests/golden/_ref/<scene>.pkl.gz``. That
folder is kept out of version control and travels with the working tree.

Usage: ``python tests/golden/make_reference_scenes.py <assets/scenes folder>`` (or set
STEEL_REFERENCE_SCENES to the folder).
"""
from __future__ import annotations

import gzip
import os
import pickle
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_ref")


def scene_names(folder: str) -> list[str]:
    return sorted(d for d in os.listdir(folder) if os.path.exists(os.path.join(folder, d, "scene.json")))


def make(folder: str, out: str = OUT) -> list[str]:
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from steel_webgpu_b200 import pack
    from steel_webgpu_b200.builder import load_scene
    os.makedirs(out, exist_ok=True)
    names = scene_names(folder)
    for name in names:
        sc = load_scene(os.path.join(folder, name))
        pk = pack(sc)
        with open(os.path.join(folder, name, "scene.json"), "rb") as f:
            text = f.read()
        tmp = os.path.join(out, name + ".pkl.gz.tmp")
        with gzip.open(tmp, "wb") as f:
            pickle.dump({"packed": pk, "json": text, "bin": sc.bin}, f, protocol=pickle.HIGHEST_PROTOCOL)
        os.replace(tmp, os.path.join(out, name + ".pkl.gz"))
    return names


if __name__ == "__main__":
    folder = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("STEEL_REFERENCE_SCENES", "")
    if not folder or not os.path.isdir(folder):
        sys.exit("give the reference's assets/scenes folder (argument or STEEL_REFERENCE_SCENES)")
    names = make(folder)
    print(f"{len(names)} scenes packed into {OUT}")
