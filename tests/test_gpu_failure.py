"""Failure paths of the step on the GPU, made without faulting it: a bounded device wait that
runs out is reported by bb_sync as BB_E_DEVICE_LIMIT, and the world steps normally afterwards.

The wait is made to run out by a block that never arrives: bb_debug_wait_limit's abandon switch
makes the last block of the colour-sweep kernel leave before its first grid barrier, and a short
wait limit (4096 polls, a few milliseconds) bounds every other block's wait for it.  Nothing
spins without a bound and no kernel traps.  Reference counterpart: the bounded walks of
avbd.slang:559, collision_detection.slang:921 and LBVH.slang:226,278, which stop without
reporting."""
import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
ERRF_SPIN_LIMIT = 1 << 2


def params(sc):
    p = bb.make_params(solver=bb.SOLVER_PGS_SOFT, iterations=8, relax_iterations=8, quirks=bb.QUIRKS_PHYSICAL)
    p.world_min[:] = sc["bounds"][0]
    p.world_extent[:] = sc["bounds"][1]
    return p


def test_a_grid_barrier_wait_that_runs_out_is_reported_and_the_world_recovers():
    sc = scenes.pile(20_000, seed=3)  # 10k items per colour at most: a colour-sweep grid of many blocks
    w = bb.world_from_scene(sc, params=params(sc))
    for _ in range(3):
        w.step(DT, 4)
    w.sync()
    assert w.stats()["manifold_count"] > 1000
    w.debug_wait_limit(4096, abandon_block=True)
    w.step(DT, 1)
    with pytest.raises(bb.BeatboxError) as e:
        w.sync()
    assert e.value.code == bb.E_DEVICE_LIMIT
    assert w.stats()["error_flags"] & ERRF_SPIN_LIMIT
    # the error is sticky until the world is cleared
    w.debug_wait_limit(0, abandon_block=False)
    with pytest.raises(bb.BeatboxError):
        w.sync()
    # cleared and reloaded, the world steps like a fresh one, bit for bit
    w.clear()
    w.add_scene(sc)
    w.set_params(params(sc))
    fresh = bb.world_from_scene(sc, params=params(sc))
    for _ in range(5):
        w.step(DT, 4)
        fresh.step(DT, 4)
    w.sync()
    fresh.sync()
    assert w.stats()["error_flags"] == 0
    a, b = w.read_state(), fresh.read_state()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_capacity_overflow_regrows_and_equals_a_large_world():
    """A world created with one pair per body on overlapping boxes overflows its pair capacity;
    with auto-regrow bb_sync reallocates it with more pairs per body, restores the state from
    before the steps since the last sync and runs them again, so it ends bit for bit where a
    world created with the large capacity ends."""
    sc = scenes.pyramids(n_pyramids=1, boxes_per=1000, gap=-0.002)  # every box overlaps its neighbours
    worlds = []
    for ppb in (1, 64):
        w = bb.World(sc["n"], pairs_per_body=ppb)
        w.add_scene(sc)
        w.set_params(params(sc))
        worlds.append(w)
    small, big = worlds
    small.set_auto_regrow(64)
    cap0 = small.stats()["pair_capacity"]
    for k in range(6):
        small.step(DT, 4)
        big.step(DT, 4)
        if k % 2 == 1:  # the first overflow is repaired with two steps to rerun
            small.sync()
    small.sync()
    big.sync()
    st = small.stats()
    assert st["error_flags"] == 0 and st["pair_capacity"] > cap0
    assert st["pair_count"] == big.stats()["pair_count"] > sc["n"]
    a, b = small.read_state(), big.read_state()
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    for what in ("manifolds", "contacts"):
        assert np.array_equal(small.debug_read(what), big.debug_read(what)), what


def test_overflow_without_regrow_is_still_reported():
    sc = scenes.pyramids(n_pyramids=1, boxes_per=1000, gap=-0.002)
    w = bb.World(sc["n"], pairs_per_body=1)
    w.add_scene(sc)
    w.set_params(params(sc))
    w.set_auto_regrow(2)  # a limit too low to hold the pairs
    w.step(DT, 1)
    with pytest.raises(bb.BeatboxError) as e:
        w.sync()
    assert e.value.code == bb.E_CAPACITY
