"""Frozen-pair carries of the narrow phase (k_narrow_carry).

A pair whose bodies both sleep keeps last substep's manifold.  When its slot was carried in place
the substep before as well, the carry rewrites only the contacts' warm-start counts (the other
contact fields already hold the same values in the buffer it writes); otherwise it copies every
field.  These tests check that both ways leave the same bits: a sleeping pile alone (its slots
never move, so its carries take the short way) against the same pile beside boxes that keep
landing elsewhere in the world (new pairs ahead of the pile's move its slots, so its carries go
through the search and copy every field).
"""
import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
BOUNDS = ([-40.0, -101.0, -40.0], [80.0, 160.0, 80.0])
PILE = 19  # ground + 18 boxes: the first ids of both worlds


def pile_scene(with_drops: bool):
    """The ground, a 4 x 4 grid of resting boxes and a 2-box stack (asleep after the quiet time),
    and optionally four columns of boxes dropped from up to 20 m far from the pile."""
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    g = np.arange(16)
    pos = np.stack([-2.4 + 1.6 * (g % 4), np.full(16, 0.499), -2.4 + 1.6 * (g // 4)], 1)
    pos = np.vstack([pos, [[4.0, 0.499, 0.0], [4.0, 1.498, 0.0]]])
    sb.add(pos, np.tile([0, 0, 0, 1.0], (18, 1)), np.full((18, 3), 0.5), scenes.SHAPE_BOX,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    if with_drops:
        drops = []
        for cx, cz in ((-20.0, -20.0), (20.0, -20.0), (-20.0, 20.0), (20.0, 20.0)):
            for k, y in enumerate((4.0, 9.0, 14.0, 20.0)):
                drops.append([cx + 0.3 * k, y, cz - 0.2 * k])
        drops = np.array(drops)
        q = np.tile([0.0, 0.0, 0.0, 1.0], (len(drops), 1))
        q[::2] = [0.0, np.sin(0.3), 0.0, np.cos(0.3)]  # some land on an edge and tumble
        sb.add(drops, q, np.full((len(drops), 3), 0.5), scenes.SHAPE_BOX,
               scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    sc = sb.build()
    sc["bounds"] = BOUNDS
    return sc


def pile_manifolds(w):
    """{(body_a, body_b, key): bytes of the manifold's fields and of its contacts} for the
    manifolds between pile bodies."""
    man = w.debug_read("manifolds")
    con = w.debug_read("contacts").reshape(len(man), 8)
    out = {}
    for m in range(len(man)):
        a, b = int(man["body_a"][m]), int(man["body_b"][m])
        if a >= PILE or b >= PILE:
            continue
        rec = man[m].copy()
        rec["color"] = 0  # the colour depends on the other manifolds' order; not carried data
        cc = int(man["contact_count"][m])
        out[(a, b, int(man["key"][m]))] = rec.tobytes() + con[m, :cc].tobytes()
    return out


def slot_of(w, a, b):
    pairs = w.debug_read("pairs").reshape(-1, 2)
    ids = w.debug_read("sorted_ids")
    pa, pb = ids[pairs[:, 0]], ids[pairs[:, 1]]
    hit = np.nonzero(((pa == a) & (pb == b)) | ((pa == b) & (pb == a)))[0]
    return int(hit[0]) if len(hit) else -1


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_PGS])
def test_short_carry_equals_full_copy(solver):
    p = bb.make_params(solver=solver, quirks=bb.QUIRKS_PHYSICAL, iterations=8, relax_iterations=8)
    if solver == bb.SOLVER_PGS:  # Baumgarte PGS runs on the per-island path
        p.flags = p.flags & ~bb.SIM_USE_GRAPH_COLORING
    alone = bb.world_from_scene(pile_scene(False), params=p)
    mixed = bb.world_from_scene(pile_scene(True), params=p)
    slots = set()
    for step in range(150):  # the last boxes land after about 2 s
        alone.step(DT, 4)
        mixed.step(DT, 4)
        if step % 3 == 0:
            slots.add(slot_of(mixed, 0, 1))  # ground and the first grid box
    alone.sync()
    mixed.sync()
    assert alone.stats()["error_flags"] == 0 and mixed.stats()["error_flags"] == 0
    assert alone.stats()["sleeping_count"] == 18
    assert len(slots - {-1}) >= 2, "the pile's slots never moved: the mixed world carries in place too"
    ga, gm = pile_manifolds(alone), pile_manifolds(mixed)
    assert len(ga) >= 18 and ga.keys() == gm.keys()
    for k in ga:
        assert ga[k] == gm[k], k
    # the carried contacts really are old: counts well past the steps of the fall
    con = alone.debug_read("contacts").reshape(-1, 8)
    man = alone.debug_read("manifolds")
    mask = np.arange(8)[None, :] < man["contact_count"][:, None]
    assert (con["warm_start"][mask] > 200).all()
