"""The C ABI from a plain C host (tests/c_abi_host.c, built with gcc against include/steel_b200.h
and the library): the header compiles as C, and the host-only entry points work without a device:
the quickhull, its error path and message, and packing a scene's files (written here from a
SceneBuilder scene) to the same statF/statU/art sizes as the Python packer; creating a context
without a device reports STEEL_E_NODEVICE (on a GPU box it succeeds)."""
import json
import os
import subprocess


from steel_webgpu_b200 import SceneBuilder, pack

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_host(steel, tmp_path):
    lib_dir = os.path.join(ROOT, "steel_webgpu_b200")
    exe = str(tmp_path / "c_abi_host")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c_abi_host.c"), "-o", exe, "-L", lib_dir, "-lsteel_b200",
                        f"-Wl,-rpath,{lib_dir}", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane(mu=0.6)
    for i in range(5):
        body = b.add_body(xform=[0.3 * i, 0.0, 0.2 + 0.25 * i, 0, 0, 0, 1])
        b.add_shape_box(body, hx=0.1, hy=0.1, hz=0.1)
    sc = b.finalize()
    (tmp_path / "scene.json").write_text(json.dumps(sc.json))
    (tmp_path / "scene.bin").write_bytes(sc.bin)
    out = subprocess.run([exe, str(tmp_path / "scene.json"), str(tmp_path / "scene.bin")], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = dict(line.split(" ", 1) for line in out.stdout.strip().splitlines())
    assert lines["hull"] == "8 6 square"
    rc, msg = lines["few"].split(" ", 1)
    assert int(rc) == 1 and "at least 4 distinct" in msg  # STEEL_E_INVALID
    pk = pack(sc)
    assert lines["pack"] == f"{pk.statF.size} {pk.statU.size} {pk.art.size}"
    import torch
    assert int(lines["device"]) == (0 if torch.cuda.is_available() else 6)  # STEEL_OK / STEEL_E_NODEVICE
