"""The TypeScript Sim (steel_webgpu_b200/ts/sim.ts, bun:ffi) binds only symbols the C header
declares, with the header's argument list: pointers and arrays as ptr, int as i32, uint32_t as u32,
uint64_t as u64, float as f32, the error string as cstring. Neither bun nor node is available
here, so the check reads both files; the library's exports are checked in test_abi.py."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_prototypes() -> dict:
    text = open(os.path.join(ROOT, "include", "steel_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for ret, name, params in re.findall(r"\b(int|const char\*)\s+(steel_\w+)\s*\(([^)]*)\)\s*;", text, re.S):
        params = params.strip()
        kinds = []
        if params and params != "void":
            for p in params.split(","):
                p = p.strip()
                if "*" in p or "[" in p:
                    kinds.append("ptr")
                elif p.startswith("int "):
                    kinds.append("i32")
                elif p.startswith("uint32_t"):
                    kinds.append("u32")
                elif p.startswith("uint64_t"):
                    kinds.append("u64")
                elif p.startswith("float"):
                    kinds.append("f32")
                else:
                    raise AssertionError(f"unknown parameter type in {name}: {p}")
        out[name] = ("cstring" if ret == "const char*" else "i32", kinds)
    return out


def ts_bindings() -> dict:
    text = open(os.path.join(ROOT, "steel_webgpu_b200", "ts", "sim.ts")).read()
    body = text[text.index("export const symbols = {"):text.index("} as const;")]
    out = {}
    for name, args, ret in re.findall(r"(steel_\w+):\s*\{\s*args:\s*\[([^\]]*)\],\s*returns:\s*([\w.]+)\s*\}", body):
        kinds = [a.strip() for a in args.split(",") if a.strip()]
        kinds = ["ptr" if k == "P" else k for k in kinds]
        out[name] = (ret.replace("FFIType.", ""), kinds)
    return out


def test_ts_symbols_match_the_header():
    hdr = header_prototypes()
    ts = ts_bindings()
    assert len(ts) >= 20
    for name, sig in ts.items():
        assert name in hdr, f"{name} is bound in sim.ts but not declared in the header"
        assert sig == hdr[name], f"{name}: sim.ts binds {sig}, the header declares {hdr[name]}"


def test_ts_sim_has_the_reference_methods():
    text = open(os.path.join(ROOT, "steel_webgpu_b200", "ts", "sim.ts")).read()
    for m in ("static async create", "destroy()", "reset()", "step(frames = 1, timestamps = false)", "async run(",
              "setJointTarget(", "setJointTargets(", "setJointForce(", "setBodyWrench(", "setBodyPose(",
              "setBodyTwist(", "async state()", "async poses()", "readPosesPooled()", "async stats()"):
        assert m in text, m
