"""Writes tests/golden/oracle_fixtures.npz: outputs of the CPU oracle on small seeded scenes.

The reference ships no golden vectors for its Sim.step path and cannot run here, so these fixtures
pin the oracle against its own earlier outputs (a change to any of them is a behaviour change that
must be deliberate), next to the analytic checks in tests/test_oracle_cpu.py:
  - the candidate pair set of the initial poses (sorted shape-index pairs);
  - the canonically sorted contact records after 30 frames (contact order and bits);
  - contact colors and row order of one prepare pass;
  - body poses and velocities, joint coordinates and speeds after 60 frames.

Run `python tests/golden/make_golden.py` from the repository root to regenerate.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _scenes():
    from tests import scenes
    return {"boxes16": scenes.boxes(n=16, seed=3), "mixed": scenes.mixed_prims(seed=3, n=12),
            "articulated": scenes.articulated(seed=5)}


def fixture_values(oracle) -> dict:
    from steel_webgpu_b200 import pack
    out = {}
    for name, sc in _scenes().items():
        pk = pack(sc)
        C = pk.C
        o = oracle.OracleSim(pk)
        o.collide()
        cnt = o.read("collide_counts", np.uint32)
        pairs = o.read("pairs", np.uint32)[:min(int(cnt[0]), C["MAXP"]) * 2].reshape(-1, 2)
        pairs = np.sort(pairs, axis=1)
        out[f"{name}/pairs0"] = np.ascontiguousarray(pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))])
        o.step(30)
        o.collide()
        cnt = o.read("collide_counts", np.uint32)
        nc = min(int(cnt[1]), C["MAXC"])
        out[f"{name}/contacts30"] = o.read("contacts")[:nc * 20].copy()
        o.stage(0)
        o.stage(1)
        sched = o.read("sched", np.uint32)
        nrows = int(sched[C["S_CSTART"] + C["NCOL"] + 1])
        out[f"{name}/colors30"] = sched[C["S_PCOL"]:C["S_PCOL"] + nrows].copy()
        out[f"{name}/order30"] = sched[C["S_PORD"]:C["S_PORD"] + nrows].copy()
        o2 = oracle.OracleSim(pk)
        o2.step(60)
        out[f"{name}/poses60"] = o2.body_poses().copy()
        out[f"{name}/vel60"] = o2.read("vel")[:pk.NB * 8].copy()
        art = o2.read("art")
        out[f"{name}/q60"] = art[C["A_Q"]:C["A_Q"] + pk.NQ].copy()
        out[f"{name}/qd60"] = art[C["A_QD"]:C["A_QD"] + pk.ND].copy()
    return out


if __name__ == "__main__":
    from oracle import oracle
    oracle.build()
    vals = fixture_values(oracle)
    np.savez_compressed(os.path.join(HERE, "oracle_fixtures.npz"), **vals)
    print({k: v.shape for k, v in vals.items()})
