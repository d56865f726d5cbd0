"""The reference's demo scenes on the GPU path, and checkpoints that resume bit for bit.

Known answers of the reference's own scenes (src/scene_manager.hpp):
  * scene_7, the box pool (:739-823): every one of the 432 cubes asleep, no fresh contact, max
    speed 0 -- under AVBD, the reference's default solver, with physical arithmetic;
  * scene_3 (:270-353): the 5-, 8- and 12-cube towers stay upright under AVBD;
  * scene_4 (:355-470): a cube slides down its ramp iff sqrt(mu_cube * mu_ramp) < tan(theta);
  * scenes 1, 2, 5 and 6 step without device errors and nothing falls through the floor.
A checkpoint (state image with the persistent contacts) restored into a new world steps exactly
as the saved world does: states and contacts equal bit for bit."""
import math

import numpy as np
import pytest

import beatbox as bb
from beatbox import io

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def params(solver, sc):
    p = bb.default_params()
    p.solver = solver
    p.quirks = bb.QUIRKS_PHYSICAL
    if solver == bb.SOLVER_PGS_SOFT:
        p.iterations = p.relax_iterations = 8
    if sc.get("bounds") is not None:
        p.world_min[:] = sc["bounds"][0]
        p.world_extent[:] = sc["bounds"][1]
    return p


def world(k, solver, pairs_per_body=16):
    sc = io.load_reference_scene(k)
    return bb.world_from_scene(sc, params=params(solver, sc), pairs_per_body=pairs_per_body), sc


def test_box_pool_falls_completely_asleep():
    w, sc = world(7, bb.SOLVER_AVBD)
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    done = None
    for step in range(900):
        w.step(DT, 4)
        if step % 10 == 9:
            st = w.stats()
            if st["sleeping_count"] == 432 and st["fresh_contacts"] == 0:
                v = w.read_state()["vel"][dyn]
                if np.sqrt((v.astype(np.float64) ** 2).sum(1)).max() == 0.0:
                    done = step
                    break
    assert done is not None, w.stats()
    assert w.stats()["error_flags"] == 0
    # everything rests on the floor or on other cubes (under full gravity some cubes land at
    # about 29 m/s and are thrown over the 10 m walls: the oracle's run shows the same)
    assert (w.read_state()["pos"][dyn, 1] > 0.4).all()


def test_towers_stay_upright():
    w, sc = world(3, bb.SOLVER_AVBD)
    x0 = sc["pos"][2:].copy()
    for _ in range(240):
        w.step(DT, 2)
    pos = w.read_state()["pos"][2:]
    assert np.abs(pos[:, [0, 2]] - x0[:, [0, 2]]).max() < 0.05
    tops = np.cumsum([5, 8, 12]) - 1
    assert np.all(pos[tops, 1] > np.array([4.5, 7.5, 11.5]) - 0.1)
    assert w.stats()["error_flags"] == 0


@pytest.mark.parametrize("solver", [bb.SOLVER_AVBD, bb.SOLVER_PGS_SOFT])
def test_cubes_slide_iff_friction_is_below_the_slope(solver):
    w, sc = world(4, solver)
    p0 = sc["pos"].copy()
    for _ in range(120):
        w.step(DT, 2)
    pos = w.read_state()["pos"]
    cubes = np.arange(4, sc["n"])
    steep = pos[cubes, 0] > 0  # the 30 degree ramp is at +x
    theta = np.where(p0[cubes, 0] > 0, math.radians(30.0), math.radians(15.0))
    mu_eff = np.sqrt(sc["friction"][cubes].astype(np.float64) * 1.0)
    moved = np.linalg.norm(pos[cubes] - p0[cubes], axis=1)
    slides = mu_eff < np.tan(theta)
    assert slides.sum() == 6 and steep.any()
    assert (moved[slides] > 0.5).all(), moved
    assert (moved[~slides] < 0.05).all(), moved
    assert w.stats()["error_flags"] == 0


@pytest.mark.parametrize("k", [1, 2, 5, 6])
def test_other_scenes_step_cleanly(k):
    w, sc = world(k, bb.SOLVER_AVBD, pairs_per_body=64 if k in (5, 6) else 16)
    for _ in range(120):
        w.step(DT, 4)
    w.sync()
    assert w.stats()["error_flags"] == 0
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    assert w.stats()["manifold_count"] > 0
    assert (w.read_state()["pos"][dyn, 1] > -0.1).all()  # nothing through the floor (top at y = 0)


@pytest.mark.parametrize("k,solver", [(7, bb.SOLVER_AVBD), (7, bb.SOLVER_PGS_SOFT), (5, bb.SOLVER_PGS_SOFT)])
def test_checkpoint_resumes_bit_for_bit(tmp_path, k, solver):
    ppb = 64 if k == 5 else 16
    w, sc = world(k, solver, pairs_per_body=ppb)
    for _ in range(60):
        w.step(DT, 4)
    path = str(tmp_path / "ck.npz")
    io.save_checkpoint(w, sc, path, pairs_per_body=ppb)
    r, sc2 = io.restore_world(path)
    assert sc2["n"] == sc["n"]
    for _ in range(20):
        w.step(DT, 4)
        r.step(DT, 4)
    w.sync()
    r.sync()
    a, b = w.read_state(), r.read_state()
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    for what in ("manifolds", "contacts"):
        assert np.array_equal(w.debug_read(what), r.debug_read(what)), what
    assert w.stats()["manifold_count"] > 0 and r.stats()["error_flags"] == 0
