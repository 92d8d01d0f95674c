"""Parity of the CUDA path with the CPU oracle on the same packed scenes.

Integer and order outputs (pair sets, the canonical contact order, colors) must match exactly;
the float pipeline is pinned to IEEE operations in a fixed order on both sides (no FMA), so
contact records, rows, poses and velocities are compared bit for bit as well.
"""
import functools

import numpy as np
import pytest

from steel_webgpu_b200 import pack
from steel_webgpu_b200.sim import Batch
from tests import scenes

pytestmark = pytest.mark.gpu

SCENES = {"boxes": scenes.boxes, "mixed_prims": scenes.mixed_prims, "articulated": scenes.articulated,
          "chains_and_quads": scenes.chains_and_quads, "hull_bin": scenes.hull_bin, "vel_limited": scenes.vel_limited,
          "chains_and_quads_fp64": scenes.chains_and_quads, "momentum_stack": scenes.momentum_stack,
          "spinners": scenes.spinners, "compliant": scenes.compliant,
          "velocity_pass": scenes.velocity_pass, "load_friction": scenes.load_friction,
          "articulated_drive_rows": scenes.articulated, "vel_limited_drive_rows": scenes.vel_limited,
          "boxes_bisection": scenes.boxes, "mixed_desaxce": scenes.mixed_prims,
          "articulated_coulomb_newton": scenes.articulated, "spin_roll": scenes.spin_roll,
          "ang_art_elliptic": scenes.ang_art,
          "ang_art_pyramid_creep": functools.partial(scenes.ang_art, cone="pyramidal", creep=0.01),
          "ang_art_relaxed": functools.partial(scenes.ang_art, relaxation=0.8),
          "four_bar": scenes.four_bar, "four_bar_cti": scenes.four_bar, "articulated_cti": scenes.articulated,
          "vel_limited_cti": scenes.vel_limited, "spin_roll_longest_first": scenes.spin_roll,
          "spinners_longest_first": scenes.spinners, "articulated_longest_first": scenes.articulated,
          "mimic_arms": scenes.mimic_arms, "mimic_arms_cti": scenes.mimic_arms}
# Packing options per scene: the FP64 articulated-inertia option on the articulation workload, PD
# drives as solver rows (drive_mode "rows"; with velocity limits, the fused drive clamp), the three
# coupled friction modes, and row_schedule "contact_then_internal" (all contact iterations, then
# the joint-internal ones) on scenes with a loop closure, limits and velocity limits, and
# propagation_color_order "longest_first" (rows colored by row count first; with contact torsion
# on `spinners`). The
# articulated torsional/rolling scenes carry their options in the scene: the elliptic cone, the
# pyramidal cone with creep compliance, and relaxation 0.8.
OPTS = {"chains_and_quads_fp64": {"solver": {"articulation_fp64": True}},
        "articulated_drive_rows": {"solver": {"drive_mode": "rows"}},
        "vel_limited_drive_rows": {"solver": {"drive_mode": "rows"}},
        "boxes_bisection": {"solver": {"friction_mode": "bisection"}},
        "mixed_desaxce": {"solver": {"friction_mode": "bisection_desaxce"}},
        "articulated_coulomb_newton": {"solver": {"friction_mode": "coulomb_newton"}},
        "four_bar_cti": {"solver": {"row_schedule": "contact_then_internal"}},
        "articulated_cti": {"solver": {"row_schedule": "contact_then_internal"}},
        "vel_limited_cti": {"solver": {"row_schedule": "contact_then_internal"}},
        "spin_roll_longest_first": {"solver": {"propagation_color_order": "longest_first"}},
        "spinners_longest_first": {"solver": {"propagation_color_order": "longest_first"}},
        "articulated_longest_first": {"solver": {"propagation_color_order": "longest_first"}},
        "mimic_arms_cti": {"solver": {"row_schedule": "contact_then_internal"}}}


def _pair_set(p):
    return {(int(min(a, b)), int(max(a, b))) for a, b in p}


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("name", ["boxes", "mixed_prims", "articulated", "hull_bin"])
def test_pairs_and_sorted_contacts(name, steel, oracle_lib):
    pk = pack(SCENES[name]())
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    for frames in (0, 30, 60):
        if frames:
            o.step(30)
            g.step(30)
        o.collide()
        g.collide()
        cnt = o.read("collide_counts", np.uint32)
        op = o.read("pairs", np.uint32)[:min(cnt[0], pk.C["MAXP"]) * 2].reshape(-1, 2)
        assert _pair_set(g.pairs()) == _pair_set(op), f"pair set differs after {frames} frames"
        nc = min(cnt[1], pk.C["MAXC"])
        rec, smu = g.contacts()
        oc = o.read("contacts")
        assert rec.shape[0] == nc
        assert np.array_equal(_bits(rec.reshape(-1)), _bits(oc[:nc * 20])), "contact records differ"
        assert np.array_equal(_bits(smu.reshape(-1)), _bits(oc[pk.C["MAXC"] * 20:pk.C["MAXC"] * 20 + nc * 4]))


@pytest.mark.parametrize("name", list(SCENES))
def test_trajectory_bit_exact(name, steel, oracle_lib):
    pk = pack(SCENES[name](), opts=OPTS.get(name))
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    nb = pk.NB
    for chunk in range(4):
        o.step(15)
        g.step(15)
        op = o.read("poses")[:nb * 8]
        gp = g.poses()
        if not np.array_equal(_bits(op), _bits(gp)):
            pytest.fail(f"{name}: poses differ after {(chunk + 1) * 15} frames (max |d| {np.abs(op - gp).max():g})")
        _, gv, gq, gqd, _ = g.raw_state()
        assert np.array_equal(_bits(o.read("vel")[:nb * 8]), _bits(gv)), "velocities differ"
        oa = o.read("art")
        assert np.array_equal(_bits(oa[pk.C["A_Q"]:pk.C["A_Q"] + pk.NQ]), _bits(gq)), "joint coordinates differ"
        assert np.array_equal(_bits(oa[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND]), _bits(gqd)), "joint velocities differ"
    ost = o.read("stats", np.uint32)
    gst = g.stats()
    assert (gst["contacts"], gst["colors"], gst["max_pairs"], gst["max_units"]) == (ost[5], ost[6], ost[4], ost[3])


@pytest.mark.parametrize("name", ["boxes", "articulated"])
def test_stage_by_stage(name, steel, oracle_lib):
    """Each substep's colors, rows and state agree after every kernel, warm-table parity included."""
    pk = pack(SCENES[name]())
    C = pk.C
    R = C["ROWS"]
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    for sub in range(40):
        o.stage(0)
        g.debug_stage(0)
        o.stage(1)
        g.debug_stage(1)
        osch = o.read("sched", np.uint32)
        nu = osch[C["S_META"]]
        tot = osch[C["S_USTART"] + nu]
        assert g.read_words("sched", g.layout("S_META"), 2, dtype=np.uint32).tolist() == [nu, osch[C["S_META"] + 1]]
        gcol = g.read_words("sched", g.layout("S_PCOL"), tot, dtype=np.uint32)
        assert np.array_equal(gcol, osch[C["S_PCOL"]:C["S_PCOL"] + tot]), f"colors differ at substep {sub}"
        assert np.array_equal(_bits(g.read_words("rows", 0, tot * R * 4)), _bits(o.read("rows")[:tot * R * 4])), \
            f"rows differ at substep {sub}"
        if pk.NL:
            assert np.array_equal(_bits(g.read_words("art", g.layout("A_LINK"), pk.NL * 268)),
                                  _bits(o.read("art")[C["A_LINK"]:C["A_LINK"] + pk.NL * 268]))
        o.stage(2)
        g.debug_stage(2)
        assert np.array_equal(_bits(g.poses()), _bits(o.read("poses")[:pk.NB * 8])), f"poses differ at substep {sub}"


def test_batch_matches_each_scene_alone(steel, oracle_lib):
    """Scenes stepped together in one batch give the same bits as each scene alone on the oracle."""
    pks = [pack(s) for s in scenes.small_batch()]
    g = Batch(pks)
    orcs = [oracle_lib.OracleSim(pk) for pk in pks]
    g.step(40)
    for i, (pk, o) in enumerate(zip(pks, orcs)):
        o.step(40)
        assert np.array_equal(_bits(g.poses(i)), _bits(o.read("poses")[:pk.NB * 8])), f"scene {i} differs"


def test_fp64_and_fp32_scenes_in_one_batch(steel, oracle_lib):
    """A batch with an ART_F64 scene runs the FP64 kernel instances; its FP32 scenes must still match
    their oracle bit for bit, and the FP64 scene its own."""
    pks = [pack(scenes.chains_and_quads(n_quad=2), opts={"solver": {"articulation_fp64": True}}),
           pack(scenes.chains_and_quads(n_quad=2)), pack(scenes.articulated())]
    assert [pk.C["ART_F64"] for pk in pks] == [1, 0, 0]
    g = Batch(pks)
    orcs = [oracle_lib.OracleSim(pk) for pk in pks]
    g.step(40)
    for i, (pk, o) in enumerate(zip(pks, orcs)):
        o.step(40)
        assert np.array_equal(_bits(g.poses(i)), _bits(o.read("poses")[:pk.NB * 8])), f"scene {i} differs"
    assert not np.array_equal(_bits(g.poses(0)), _bits(g.poses(1))), "the option changed nothing"


def test_extended_solve_instance_in_a_mixed_batch(steel, oracle_lib):
    """A batch with an articulated torsional/rolling scene or a contact-then-internal scene runs the
    extended solve instance for all its scenes; the plain scenes in it (and a longest-first one)
    must still match their oracle bit for bit."""
    pks = [pack(scenes.ang_art()), pack(scenes.four_bar(), opts={"solver": {"row_schedule": "contact_then_internal"}}),
           pack(scenes.articulated()), pack(scenes.spin_roll(), opts={"solver": {"propagation_color_order": "longest_first"}}),
           pack(scenes.mimic_arms())]
    assert (pks[0].C["ANG_ART"], pks[1].C["CTI"], pks[3].C["LONGEST_FIRST"]) == (1, 1, 1)
    g = Batch(pks)
    orcs = [oracle_lib.OracleSim(pk) for pk in pks]
    g.step(40)
    for i, (pk, o) in enumerate(zip(pks, orcs)):
        o.step(40)
        assert np.array_equal(_bits(g.poses(i)), _bits(o.read("poses")[:pk.NB * 8])), f"scene {i} differs"
        if pk.NQ:
            _, _, gq, gqd, _ = g.raw_state(i)
            oa = o.read("art")
            assert np.array_equal(_bits(gqd), _bits(oa[pk.C["A_QD"]:pk.C["A_QD"] + pk.ND])), f"scene {i} qd differs"


def test_sleeping_bit_exact(steel, oracle_lib):
    """Islands fall asleep, wake on contact and sleep again identically: poses, velocities, joint
    state, per-node (age, asleep) words and the asleep count every 20 frames over 320 frames."""
    pk = pack(scenes.sleepers())
    assert pk.C["SLEEP"] == 1
    o = oracle_lib.OracleSim(pk)
    g = Batch([pk])
    nn = pk.NB + pk.NA
    counts = []
    for k in range(16):
        o.step(20)
        g.step(20)
        oa = o.read("art")
        assert np.array_equal(_bits(g.poses()), _bits(o.read("poses")[:pk.NB * 8])), f"poses differ at {20 * (k + 1)}"
        _, gv, gq, gqd, _ = g.raw_state()
        assert np.array_equal(_bits(gv), _bits(o.read("vel")[:pk.NB * 8]))
        assert np.array_equal(_bits(gq), _bits(oa[pk.C["A_Q"]:pk.C["A_Q"] + pk.NQ]))
        gslp = g.read_words("art", g.layout("A_SLP"), nn * 4)
        assert np.array_equal(_bits(gslp), _bits(oa[pk.C["A_SLP"]:pk.C["A_SLP"] + nn * 4])), "sleep words differ"
        ost = o.read("stats", np.uint32)
        assert g.stats()["asleep"] == int(ost[8])
        counts.append(int(ost[8]))
    # Asleep, woken by the dropped box, asleep again.
    first = next(i for i, c in enumerate(counts) if c >= 6)
    assert min(counts[first:]) < counts[first] and counts[-1] >= 6, counts


def test_block_size_does_not_change_results(steel):
    """A batch of no more scenes than SMs runs prepare and solve with 512-thread blocks, a larger
    batch with 128-thread blocks; the same scene gives the same bits either way."""
    pk = pack(scenes.chains_and_quads(n_quad=2))
    small = Batch([pk])
    large = Batch([pk] * 160)
    small.step(20)
    large.step(20)
    for i in (0, 159):
        assert np.array_equal(_bits(small.poses()), _bits(large.poses(i)))
        assert np.array_equal(_bits(small.raw_state()[2]), _bits(large.raw_state(i)[2]))


@pytest.mark.parametrize("tiles", [(128, 0, 0, 1), (128, 54000, 0, 1), (64, 25000, 0, 1), (64, 6000, 0, 1),
                                   (32, 11000, 0, 1), (32, 2000, 1, 1), (64, 12928, 0, 2), (128, 0, 0, 3)])
def test_tiles_do_not_change_results(tiles, steel):
    """Every tile configuration (block size, shared-memory staging budget, narrowphase grid, scene
    groups on parallel streams) gives the same bits as the default, for a batch with more scenes
    than SMs (uneven scenes with chains, quadrupeds and a plain box pile)."""
    pks = [pack(s) for s in scenes.small_batch(n=6)] + [pack(scenes.chains_and_quads(n_quad=2)),
                                                          pack(scenes.articulated()), pack(scenes.boxes(40))]
    pks = pks * 17  # 153 scenes > 148 SMs
    ref = Batch(pks)
    g = Batch(pks)
    assert ref.tiles()["block_threads"] == 128
    g.set_tiles(*tiles)
    assert g.tiles() == dict(block_threads=tiles[0], smem_budget=tiles[1], narrow_blocks_per_sm=tiles[2],
                             stream_groups=tiles[3])
    ref.step(20)
    g.step(20)
    for i in (0, 1, 5, 6, 7, 8, 76, 77, 150, 152):
        assert np.array_equal(_bits(ref.poses(i)), _bits(g.poses(i))), f"scene {i} differs under {tiles}"
        assert np.array_equal(_bits(ref.raw_state(i)[3]), _bits(g.raw_state(i)[3]))


@pytest.mark.parametrize("threads", [512, 256, 64, 32])
def test_tiles_of_a_single_large_scene(threads, steel):
    """A batch of one scene starts at 512-thread blocks; every smaller block gives the same bits."""
    pk = pack(scenes.chains_and_quads(n_quad=6))
    ref = Batch([pk])
    g = Batch([pk])
    assert ref.tiles()["block_threads"] == 512
    g.set_tiles(threads, 0 if threads >= 256 else 20000)
    ref.step(20)
    g.step(20)
    assert np.array_equal(_bits(ref.poses()), _bits(g.poses()))
    assert np.array_equal(_bits(ref.raw_state()[2]), _bits(g.raw_state()[2]))


def test_autotune_picks_a_config_and_resets(steel, oracle_lib):
    """The autotuner times its candidates, keeps one and resets the batch: stepping afterwards
    matches the oracle from the initial state."""
    pks = [pack(s) for s in scenes.small_batch(n=6)]
    g = Batch(pks)
    g.step(5)
    tiles, ms = g.autotune(2)
    assert tiles["block_threads"] in (32, 64, 128, 256, 512) and ms > 0
    assert g.tiles() == tiles
    g.step(20)
    for i, pk in enumerate(pks):
        o = oracle_lib.OracleSim(pk)
        o.step(20)
        assert np.array_equal(_bits(g.poses(i)), _bits(o.read("poses")[:pk.NB * 8])), f"scene {i} differs"


def test_tiles_reject_bad_values(steel):
    pks = [pack(scenes.boxes(8))] * 200
    g = Batch(pks)
    from steel_webgpu_b200 import _lib
    for bad in ((512, 0, 0), (96, 0, 0), (128, 0, 99), (128, 0, 0, 9)):
        with pytest.raises(_lib.SteelError):
            g.set_tiles(*bad)


def test_reset_replays_identically(steel):
    pk = pack(scenes.boxes(24))
    g = Batch([pk])
    g.step(30)
    a = g.poses().copy()
    g.reset()
    g.step(30)
    assert np.array_equal(_bits(a), _bits(g.poses()))


def test_graph_and_eager_launches_agree(steel):
    pk = pack(scenes.articulated())
    g1 = Batch([pk], graph=True)
    g2 = Batch([pk], graph=False)
    g1.step(20)
    g2.step(20)
    assert np.array_equal(_bits(g1.poses()), _bits(g2.poses()))


def test_batches_with_different_shared_memory_coexist(steel):
    """A kernel's largest dynamic shared memory is set for the whole process: a batch created
    after another, with smaller staging needs, must not break the first one's launches (graph
    capture included)."""
    big = Batch([pack(scenes.chains_and_quads(n_quad=2))] * 3)
    small = Batch([pack(scenes.boxes(8))] * 3)
    small.step(2)
    big.step(2)
    big.sync()
    ref = Batch([pack(scenes.chains_and_quads(n_quad=2))])
    ref.step(2)
    assert np.array_equal(_bits(big.poses(1)), _bits(ref.poses()))
