"""The team solve (steel_set_team): a batch of one scene solved by a cooperative launch of several
blocks that meet at grid barriers gives the same bits as the one-block solve.

Covered: every option scene of the parity tests forced onto a small team (Nesterov momentum keeps
one block), a pour large enough for the default rule (with and without the frame graph), an
articulation scene with more articulations than the rule's threshold, and the rule's edges
(batches of several scenes and small scenes keep one block; a request for more blocks than fit is
refused).
"""
import numpy as np
import pytest

from steel_webgpu_b200 import pack, synth
from steel_webgpu_b200._lib import SteelError
from steel_webgpu_b200.sim import Batch, auto_caps
from tests import scenes
from tests.test_parity_gpu import OPTS, SCENES

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32).copy()


def _run(pk, team, frames, graph=True):
    """Steps a one-scene batch with the given team request; returns (blocks used, state bits, stats)."""
    g = Batch([pk], graph=graph)
    g.set_team(team)
    used = g.team()
    g.step(frames)
    pos, vel, q, qd, lv = g.raw_state()
    st = g.stats()
    g.close()
    return used, [_bits(x) for x in (pos, vel, q, qd, lv)], st


def _same(ref, got, what):
    for k, (a, b) in enumerate(zip(ref[1], got[1])):
        assert np.array_equal(a, b), f"{what}: {['poses', 'velocities', 'q', 'qd', 'link twists'][k]} differ"
    assert ref[2] == got[2], f"{what}: stats differ"


@pytest.mark.parametrize("name", sorted(SCENES))
def test_option_scenes_on_a_team(name, steel):
    pk = pack(SCENES[name](), opts=OPTS.get(name))
    ref = _run(pk, 0, 30)
    assert ref[0] == 0
    got = _run(pk, 3, 30)
    assert got[0] == (0 if name == "momentum_stack" else 3)  # Nesterov momentum: one block
    _same(ref, got, name)


def _pour(n, seed):
    sc = synth.convex_pour(n=n, seed=seed)
    caps = auto_caps(sc)
    caps.update(MAXP=1 << 17, MAXC=1 << 17, MAXU=1 << 17, UH=1 << 17, WH=1 << 18, AH=1 << 17)
    return pack(sc, caps=caps)


def test_pour_default_team(steel):
    """3000 bodies poured into the bin: the default rule makes a team; 3 frames match one block,
    with the frame graph and without, and on a team of 37 blocks."""
    pk = _pour(3000, 2)
    ref = _run(pk, 0, 3)
    auto = _run(pk, Batch.TEAM_AUTO, 3)
    assert auto[0] >= 2
    _same(ref, auto, "default team")
    assert ref[2]["overflow"] == []
    _same(ref, _run(pk, Batch.TEAM_AUTO, 3, graph=False), "default team, no graph")
    _same(ref, _run(pk, 37, 3), "37 blocks")


def test_articulations_default_team(steel):
    """70 PD-driven quadrupeds and 4 40-link chains (74 articulations, above the rule's 64): a warp
    per articulation over the team's blocks matches one block over 2 frames."""
    sc = synth.quadrupeds(n_quad=70, n_chains=4, chain_links=40, seed=3)
    pk = pack(sc, caps=auto_caps(sc))
    ref = _run(pk, 0, 2)
    auto = _run(pk, Batch.TEAM_AUTO, 2)
    assert auto[0] >= 2
    _same(ref, auto, "articulations on the default team")


def test_team_rule_edges(steel):
    small = pack(scenes.boxes())
    g = Batch([small])
    assert g.team() == 0  # below the default rule's size
    g.set_team(2)
    assert g.team() == 2
    with pytest.raises(SteelError):
        g.set_team(100000)
    g.close()
    two = Batch([small, small])
    two.set_team(4)
    assert two.team() == 0  # several scenes: one block per scene
    two.close()
