"""GPU parity tests: the CUDA library (through its C ABI) against the oracle.

Tolerances:
  * bit-exact: Morton codes, sorted keys and ids, LBVH topology, leaf and node boxes, pairs,
    manifold identities (bodies, SAT key, contact count), edge and body colourings;
  * narrow-phase geometry (FP32 kernel vs FP64 oracle): normals 1e-5, contact points and
    depths 1e-4 m;
  * one step from a contact-rich state: relative error <= 1e-4 of the world's scale for
    positions and 2e-4 (abs floor 2e-4 m/s) for velocities;
  * 300 steps: aggregate statistics within bands (see test_300_step_statistics).
"""
import math

import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def oracle_for(po, sc, params):
    return po.Oracle(sc, params=params)


def params_for(po, sc, **kw):
    p = po.default_params()
    for k, v in kw.items():
        setattr(p, k, v)
    if sc.get("bounds") is not None:
        p.world_min[:] = sc["bounds"][0]
        p.world_extent[:] = sc["bounds"][1]
    return p


def oread(o, code, dtype):
    cnt, buf = o.debug_read(code)
    itemsize = np.dtype(dtype).itemsize
    if code == 8:
        return buf[: cnt * bb.MANIFOLD_DTYPE.itemsize].view(bb.MANIFOLD_DTYPE)
    if code == 9:
        return buf[: cnt * bb.CONTACT_DTYPE.itemsize].view(bb.CONTACT_DTYPE)
    return buf[: cnt * itemsize].view(dtype)


def dup_scene():
    """Bodies sharing Morton cells (duplicate codes exercise the index tie-break)."""
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    pos = np.array([[0.01 * (k % 3), 0.6 + 0.02 * (k // 3), 0.0] for k in range(12)])
    sb.add(pos, np.tile([0, 0, 0, 1.0], (12, 1)), np.full((12, 3), 0.05), 0,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1.0)
    return sb.build()


def single_scene(n):
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    if n > 1:
        sb.add([[0, 0.45, 0]] * (n - 1), [[0, 0, 0, 1]] * (n - 1), [[0.5] * 3] * (n - 1), 0,
               scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1.0)
    return sb.build()


FRONT_SCENES = {
    "box_grid_1000": lambda: scenes.box_grid(),
    "mixed_2000": lambda: scenes.mixed_column(n_bodies=2000, seed=1),
    "pyramids_2x1000": lambda: scenes.pyramids(n_pyramids=2, boxes_per=1000, gap=-0.002),
    "duplicates": dup_scene,
    "one_body": lambda: single_scene(1),
    "two_bodies": lambda: single_scene(2),
}


@pytest.mark.parametrize("name", sorted(FRONT_SCENES))
@pytest.mark.parametrize("bounds", [bb.BOUNDS_FIXED, bb.BOUNDS_AUTO])
def test_front_end_bit_exact(oracle_lib, name, bounds):
    sc = FRONT_SCENES[name]()
    p = params_for(oracle_lib, sc, bounds_mode=bounds)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    w.debug_collide(1)
    o.collide(1)
    assert np.array_equal(w.debug_read("morton"), oread(o, 1, np.uint32))
    assert np.array_equal(w.debug_read("sorted_keys"), oread(o, 2, np.uint32))
    assert np.array_equal(w.debug_read("sorted_ids"), oread(o, 3, np.uint32))
    assert np.array_equal(w.debug_read("lbvh_child"), oread(o, 4, np.int32))
    assert np.array_equal(w.debug_read("leaf_aabb"), oread(o, 5, np.float32))
    assert np.array_equal(w.debug_read("node_aabb"), oread(o, 6, np.float32))
    assert np.array_equal(w.debug_read("pairs"), oread(o, 7, np.uint32))
    # a second collide starts from the new sorted order on both sides
    w.debug_collide(1)
    o.collide(1)
    assert np.array_equal(w.debug_read("sorted_ids"), oread(o, 3, np.uint32))
    assert np.array_equal(w.debug_read("pairs"), oread(o, 7, np.uint32))


@pytest.mark.parametrize("name,quirks", [("box_grid_1000", 0), ("box_grid_1000", 7), ("mixed_2000", 0),
                                         ("mixed_2000", 7), ("pyramids_2x1000", 0)])
def test_narrow_phase_matches_oracle(oracle_lib, name, quirks):
    sc = FRONT_SCENES[name]()
    if name == "mixed_2000":  # drop the column onto itself so boxes and spheres touch
        sc = dict(sc)
        pos = sc["pos"].copy()
        pos[5:, 1] = 0.5 + (pos[5:, 1] - 1.0) * 0.02
        sc["pos"] = pos
    p = params_for(oracle_lib, sc, quirks=quirks)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    w.debug_collide(2)
    o.collide(2)
    gm, rm = w.debug_read("manifolds"), oread(o, 8, None)
    assert len(gm) == len(rm) and len(gm) > 0
    assert np.array_equal(gm["body_a"], rm["body_a"]) and np.array_equal(gm["body_b"], rm["body_b"])
    assert np.array_equal(gm["key"], rm["key"])
    assert np.array_equal(gm["contact_count"], rm["contact_count"])
    assert np.abs(gm["normal"] - rm["normal"]).max() < 1e-5
    gc, rc = w.debug_read("contacts"), oread(o, 9, None)
    mask = np.repeat(np.arange(8)[None, :], len(gm), 0) < gm["contact_count"][:, None]
    mask = mask.ravel()
    assert np.abs(gc["position"][mask] - rc["position"][mask]).max() < 1e-4
    assert np.abs(gc["penetration"][mask] - rc["penetration"][mask]).max() < 1e-4
    assert np.array_equal(gc["feature"][mask], rc["feature"][mask])


def settled(po, sc, solver, quirks, steps):
    """A contact-rich state: the FP64 oracle run for `steps` steps, as float32 arrays."""
    p = params_for(po, sc, solver=solver, quirks=quirks, iterations=8, relax_iterations=8, avbd_iterations=4)
    o = oracle_for(po, sc, p)
    for _ in range(steps):
        o.step(DT, 4)
    st = o.state()
    sc2 = dict(sc)
    sc2["pos"], sc2["quat"] = st["pos"].astype(np.float32), st["quat"].astype(np.float32)
    sc2["vel"], sc2["omega"] = st["vel"].astype(np.float32), st["omega"].astype(np.float32)
    sc2["flags"] = sc["flags"].copy()  # everyone awake
    return sc2, p


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
@pytest.mark.parametrize("quirks", [bb.QUIRKS_PHYSICAL, bb.QUIRKS_REFERENCE])
def test_one_step_state_within_tolerance(oracle_lib, solver, quirks):
    base = scenes.box_grid(n_side=6, layers=4, density=5.0 if solver == bb.SOLVER_AVBD else 1000.0)
    sc, p = settled(oracle_lib, base, solver, quirks, 45)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    o.step(DT, 4)
    w.step(DT, 4)
    w.sync()
    assert w.stats()["manifold_count"] > 50
    # identical colourings of the last substep (same manifolds -> same colours)
    assert np.array_equal(w.debug_read("edge_colors"), oread(o, 10, np.uint32))
    g, r = w.read_state(), o.state()
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    pos_scale = np.abs(r["pos"][dyn]).max()
    perr = np.abs(g["pos"][dyn] - r["pos"][dyn]).max() / pos_scale
    vscale = max(np.abs(r["vel"][dyn]).max(), 1.0)
    verr = np.abs(g["vel"][dyn] - r["vel"][dyn]).max()
    assert perr < 1e-4, perr
    assert verr < 2e-4 * vscale, verr


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS, bb.SOLVER_PGS_SOFT])
def test_per_island_path_one_step_within_tolerance(oracle_lib, solver):
    """USE_GRAPH_COLORING off: every contact island solved serially in manifold order, with the
    Baumgarte PGS or PGS_SOFT, against the oracle's same schedule."""
    base = scenes.box_grid(n_side=6, layers=4)
    sc, p = settled(oracle_lib, base, bb.SOLVER_PGS_SOFT, bb.QUIRKS_PHYSICAL, 45)
    p.solver = solver
    p.flags = p.flags & ~bb.SIM_USE_GRAPH_COLORING
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    o.step(DT, 4)
    w.step(DT, 4)
    w.sync()
    st = w.stats()
    assert st["manifold_count"] > 50 and st["graph_color_count"] == 0 and st["error_flags"] == 0
    g, r = w.read_state(), o.state()
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    perr = np.abs(g["pos"][dyn] - r["pos"][dyn]).max() / np.abs(r["pos"][dyn]).max()
    verr = np.abs(g["vel"][dyn] - r["vel"][dyn]).max()
    assert perr < 1e-4, perr
    assert verr < 2e-4 * max(np.abs(r["vel"][dyn]).max(), 1.0), verr


def test_per_island_pgs_settles_a_pile():
    sc = scenes.box_grid(n_side=5, layers=3)
    p = bb.make_params(solver=bb.SOLVER_PGS, quirks=bb.QUIRKS_PHYSICAL, iterations=8, relax_iterations=8)
    p.flags = p.flags & ~bb.SIM_USE_GRAPH_COLORING
    w = bb.world_from_scene(sc, params=p)
    for _ in range(180):
        w.step(DT, 4)
    st = w.read_state()
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    assert np.abs(st["vel"][dyn]).max() < 0.5
    assert st["pos"][dyn, 1].min() > 0.3  # resting on the ground, nothing fell through
    assert w.stats()["error_flags"] == 0


def energy_stats(state, sc):
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    m = sc["mass"][dyn].astype(np.float64)
    v = state["vel"][dyn].astype(np.float64)
    y = state["pos"][dyn, 1].astype(np.float64)
    return dict(ke=float(0.5 * (m * (v ** 2).sum(1)).sum()), pe=float((m * 9.81 * y).sum()),
                mom=float(np.abs((m[:, None] * v).sum(0)).sum()), ymean=float(y.mean()))


def quat_matrix(q):
    x, y, z, w = (q[:, k] for k in range(4))
    return np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], 1),
                     np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], 1),
                     np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1)], 1)


def dynamics(state, sc):
    """Total linear momentum P, angular momentum L about the dynamic bodies' centre of mass,
    and energy E = kinetic (linear + rotational) + potential (g = 9.81 m/s^2)."""
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    m = sc["mass"][dyn].astype(np.float64)
    x = state["pos"][dyn].astype(np.float64)
    v = state["vel"][dyn].astype(np.float64)
    w = state["omega"][dyn].astype(np.float64)
    ii = sc["inv_inertia"][dyn].astype(np.float64)
    inertia = np.where(ii > 0, 1.0 / np.where(ii > 0, ii, 1.0), 0.0)  # body-frame diagonal
    R = quat_matrix(state["quat"][dyn].astype(np.float64))
    wb = np.einsum("nji,nj->ni", R, w)  # angular velocity in the body frame
    com = (m[:, None] * x).sum(0) / m.sum()
    P = (m[:, None] * v).sum(0)
    L = (np.cross(x - com, m[:, None] * v) + np.einsum("nij,nj->ni", R, inertia * wb)).sum(0)
    E = 0.5 * (m * (v ** 2).sum(1)).sum() + 0.5 * (inertia * wb ** 2).sum() + (m * 9.81 * x[:, 1]).sum()
    return P, L, E


def mean_penetration(manifolds, contacts):
    mask = (np.arange(8)[None, :] < manifolds["contact_count"][:, None]).ravel()
    pen = contacts["penetration"][mask]
    pen = pen[pen < 0]
    return float(pen.mean()) if len(pen) else 0.0


def test_300_step_statistics(oracle_lib):
    """1,000-box grid, PGS 8 iterations, 4 substeps, 300 steps: GPU (FP32) vs oracle (FP64).
    The trajectories are chaotic, so statistics are compared, every step, within bands set
    several times wider than the oracle's own FP32 build lands from its FP64 build:
      * total linear momentum within 2% of M g (1 s) (M: the pile's mass);
      * angular momentum about the pile's centre of mass within 2% of M g (1 s) R0 (R0: the
        grid's RMS radius about that centre at the start);
      * energy (kinetic + potential) within 5% of the energy the oracle's run dissipates;
      * mean penetration of the penetrating contacts, averaged over steps 100..299, within 1 mm;
    and at the end: mean height within 2 cm, potential energy within 1%, max penetration within
    1 cm, sleeping count within 100, kinetic energy small on both."""
    sc = scenes.box_grid()
    p = params_for(oracle_lib, sc, solver=1, quirks=0, iterations=8, relax_iterations=8)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    M = float(sc["mass"][dyn].sum())
    x0 = sc["pos"][dyn].astype(np.float64)
    R0 = float(np.sqrt(((x0 - x0.mean(0)) ** 2).sum(1).mean()))
    E0 = dynamics(o.state(), sc)[2]
    dP, dL, dE, pen_g, pen_r = [], [], [], [], []
    for k in range(300):
        w.step(DT, 4)
        o.step(DT, 4)
        Pg, Lg, Eg = dynamics(w.read_state(), sc)
        Pr, Lr, Er = dynamics(o.state(), sc)
        dP.append(np.abs(Pg - Pr).max())
        dL.append(np.abs(Lg - Lr).max())
        dE.append(abs(Eg - Er))
        if k >= 100:
            pen_g.append(mean_penetration(w.debug_read("manifolds"), w.debug_read("contacts")))
            pen_r.append(mean_penetration(oread(o, 8, None), oread(o, 9, None)))
    w.sync()
    dissipated = E0 - Er
    assert dissipated > 0
    assert max(dP) <= 0.02 * M * 9.81, (max(dP), M * 9.81)
    assert max(dL) <= 0.02 * M * 9.81 * R0, (max(dL), M * 9.81 * R0)
    assert max(dE) <= 0.05 * dissipated, (max(dE), dissipated)
    assert abs(np.mean(pen_g) - np.mean(pen_r)) <= 1e-3, (np.mean(pen_g), np.mean(pen_r))
    g, r = energy_stats(w.read_state(), sc), energy_stats(o.state(), sc)
    gs, rs = w.stats(), o.stats()
    assert abs(g["ymean"] - r["ymean"]) < 0.02
    assert abs(g["pe"] - r["pe"]) / r["pe"] < 0.01
    assert abs(gs["max_penetration"] - rs["max_penetration"]) < 0.01
    assert abs(gs["sleeping_count"] - rs["sleeping_count"]) <= 100
    assert g["ke"] < 1e-2 * r["pe"] and r["ke"] < 1e-2 * r["pe"]
    assert gs["error_flags"] == 0 and gs["graph_color_overflow"] == 0


def test_steps_are_deterministic(oracle_lib):
    sc = scenes.mixed_column(n_bodies=3000, seed=2)
    outs = []
    for _ in range(2):
        p = params_for(oracle_lib, sc, solver=1, quirks=0)
        w = bb.world_from_scene(sc, params=p)
        for _ in range(40):
            w.step(DT, 4)
        outs.append(w.read_state())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k])


def test_avbd_colouring_valid_and_matches_oracle(oracle_lib):
    sc = scenes.box_grid(n_side=6, layers=4, density=5.0)
    sc2, p = settled(oracle_lib, sc, bb.SOLVER_AVBD, 0, 30)
    w = bb.world_from_scene(sc2, params=p)
    o = oracle_for(oracle_lib, sc2, p)
    w.step(DT, 1)
    o.step(DT, 1)
    gcol, rcol = w.debug_read("body_colors"), oread(o, 11, np.uint32)
    assert np.array_equal(gcol, rcol)
    st = w.stats()
    assert st["avbd_color_count"] == o.stats()["avbd_color_count"] > 0
    # validity: no manifold joins two dynamic bodies of the same colour
    man = w.debug_read("manifolds")
    dyn = (sc2["flags"] & bb.BODY_DYNAMIC) != 0
    both = dyn[man["body_a"]] & dyn[man["body_b"]]
    assert np.all(gcol[man["body_a"][both]] != gcol[man["body_b"][both]])


def test_capacity_overflow_is_reported(oracle_lib):
    # overlapping boxes: every box pairs with up to 26 neighbours, far above one pair per body
    sc = scenes.pyramids(n_pyramids=1, boxes_per=1000, gap=-0.002)
    w = bb.World(sc["n"], pairs_per_body=1)
    w.add_scene(sc)
    w.step(DT, 1)
    with pytest.raises(bb.BeatboxError) as e:
        w.sync()
    assert e.value.code == bb.E_CAPACITY


def test_invalid_arguments_are_rejected():
    w = bb.World(8)
    with pytest.raises(bb.BeatboxError) as e:
        w.step(0.0, 1)
    assert e.value.code == bb.E_INVALID
    with pytest.raises(bb.BeatboxError) as e:  # Baumgarte PGS runs on the per-island path only
        w.set_params(solver=bb.SOLVER_PGS)
    assert e.value.code == bb.E_INVALID
    with pytest.raises(bb.BeatboxError):
        w.add_box_shape(-1.0, 1.0, 1.0)


def test_rigid_body_manager_facade():
    m = bb.RigidBodyManager(max_bodies=64)
    assert m.create("test", iterations=6)
    sc = scenes.box_grid(n_side=3, layers=2)
    m.world.add_scene(sc)
    m.set_sim_type(bb.SOLVER_PGS_SOFT)
    m.clear_sim_flags(bb.SIM_SLEEPING_ENABLED)
    assert not (m.get_sim_flags() & bb.SIM_SLEEPING_ENABLED)
    for _ in range(10):
        assert m.simulate()
    assert m.read_back_sim_config()
    cfg = m.get_sim_config_reference()
    assert cfg["body_count"] == sc["n"] and cfg["error_flags"] == 0


def test_state_roundtrip_and_write():
    sc = scenes.box_grid(n_side=3, layers=2)
    w = bb.world_from_scene(sc)
    st = w.read_state()
    assert np.allclose(st["pos"], sc["pos"]) and np.allclose(st["quat"], sc["quat"])
    newpos = st["pos"] + 1.0
    w.write_state(pos=newpos)
    assert np.allclose(w.read_state()["pos"], newpos)


def resting_scene():
    """Boxes resting on the ground from the start (a 4 x 4 grid of singles and one 2-box stack):
    they fall asleep after the quiet-time threshold, on the GPU and in the oracle alike."""
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    g = np.arange(16)
    pos = np.stack([-2.4 + 1.6 * (g % 4), np.full(16, 0.499), -2.4 + 1.6 * (g // 4)], 1)
    pos = np.vstack([pos, [[4.0, 0.499, 0.0], [4.0, 1.498, 0.0]]])
    sb.add(pos, np.tile([0, 0, 0, 1.0], (18, 1)), np.full((18, 3), 0.5), scenes.SHAPE_BOX,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    return sb.build()


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_PGS])
def test_sleeping_bodies_carry_their_manifolds_like_the_oracle(oracle_lib, solver):
    """Bodies that fall asleep during the run: from the second substep they sleep, their frozen
    pairs carry their manifolds over (impulses, features, warm-start counts + 1) on both sides.
    Sleep counts, manifold identities, features and warm-start counts match the oracle bit for
    bit, and the sleeping bodies do not move."""
    sc = resting_scene()
    p = params_for(oracle_lib, sc, solver=solver, quirks=0, iterations=8, relax_iterations=8)
    if solver == bb.SOLVER_PGS:  # Baumgarte PGS runs on the per-island path
        p.flags = p.flags & ~bb.SIM_USE_GRAPH_COLORING
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    for _ in range(50):
        w.step(DT, 4)
        o.step(DT, 4)
    before = w.read_state()
    for _ in range(10):
        w.step(DT, 4)
        o.step(DT, 4)
    w.sync()
    gs, rs = w.stats(), o.stats()
    assert gs["sleeping_count"] == rs["sleeping_count"] == 18
    gm, rm = w.debug_read("manifolds"), oread(o, 8, None)
    assert len(gm) == len(rm) == 18
    for f in ("body_a", "body_b", "key", "contact_count"):
        assert np.array_equal(gm[f], rm[f]), f
    gc, rc = w.debug_read("contacts"), oread(o, 9, None)
    mask = (np.arange(8)[None, :] < gm["contact_count"][:, None]).ravel()
    assert np.array_equal(gc["feature"][mask], rc["feature"][mask])
    assert np.array_equal(gc["warm_start"][mask], rc["warm_start"][mask])
    assert (gc["warm_start"][mask] > 200).all()  # every contact inherited since the first substeps
    assert np.abs(gc["position"][mask] - rc["position"][mask]).max() < 1e-4
    after = w.read_state()
    for k in before:
        assert np.array_equal(before[k], after[k]), k  # asleep: frozen in place


def test_resting_islands_are_left_uncoloured(oracle_lib):
    """The 18 boxes of the resting scene fall asleep while a three-box stack is in free fall
    elsewhere.  The edge colouring skips the islands with no awake body (their manifolds read
    EDGE_COLOR_RESTING and are not solved); every other manifold keeps the colour the oracle,
    which colours all manifolds, gives it, because the colouring rounds are local to an island."""
    sc = resting_scene()
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    sb.add(sc["pos"][1:], sc["quat"][1:], sc["half"][1:], scenes.SHAPE_BOX,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    stack = np.array([[12.0, 5.0, 0.0], [12.0, 5.999, 0.0], [12.0, 6.998, 0.0]])
    sb.add(stack, np.tile([0, 0, 0, 1.0], (3, 1)), np.full((3, 3), 0.5), scenes.SHAPE_BOX,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    sc = sb.build()
    p = params_for(oracle_lib, sc, solver=bb.SOLVER_PGS_SOFT, quirks=0, iterations=8, relax_iterations=8)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    for _ in range(20):
        w.step(DT, 4)
        o.step(DT, 4)
    w.sync()
    assert w.stats()["sleeping_count"] == o.stats()["sleeping_count"] == 18
    gm, rm = w.debug_read("manifolds"), oread(o, 8, None)
    assert len(gm) == len(rm)
    for f in ("body_a", "body_b", "key", "contact_count"):
        assert np.array_equal(gm[f], rm[f]), f
    gcol, rcol = w.debug_read("edge_colors"), oread(o, 10, np.uint32)
    in_stack = (gm["body_a"] >= 19) | (gm["body_b"] >= 19)
    assert in_stack.sum() == 2  # the stack's two inner manifolds, sharing the middle box
    assert (gcol[~in_stack] == bb.EDGE_COLOR_RESTING).all()
    assert np.array_equal(gcol[in_stack], rcol[in_stack])
    assert sorted(gcol[in_stack].tolist()) == [0, 1]
    assert w.stats()["graph_color_count"] == 2 and w.stats()["error_flags"] == 0


def test_islands_start_from_last_roots_like_a_fresh_union_find(oracle_lib):
    """Connected components start from the last substep's roots for components whose bodies
    were not awake at two narrow phases in a row.  A three-box stack falls onto the sleeping
    two-box stack of the resting scene and wakes it; the island of every body must equal the
    oracle's union-find from scratch at every step whose manifolds agree (most of them)."""
    sc = resting_scene()
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    sb.add(sc["pos"][1:], sc["quat"][1:], sc["half"][1:], scenes.SHAPE_BOX,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    stack = np.array([[4.0, 4.0, 0.0], [4.0, 4.999, 0.0], [4.0, 5.998, 0.0]])
    sb.add(stack, np.tile([0, 0, 0, 1.0], (3, 1)), np.full((3, 3), 0.5), scenes.SHAPE_BOX,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1000.0)
    sc = sb.build()
    p = params_for(oracle_lib, sc, solver=bb.SOLVER_PGS_SOFT, quirks=0, iterations=8, relax_iterations=8)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_for(oracle_lib, sc, p)
    compared, merged, slept = 0, 0, 0
    for _ in range(70):
        w.step(DT, 4)
        o.step(DT, 4)
        w.sync()
        gm, rm = w.debug_read("manifolds"), oread(o, 8, None)
        if len(gm) != len(rm) or not all(np.array_equal(gm[f], rm[f]) for f in ("body_a", "body_b")):
            continue
        gi, ri = w.debug_read("islands"), oread(o, 12, np.uint32)
        assert np.array_equal(gi, ri)
        assert w.stats()["island_count"] == o.stats()["island_count"]
        compared += 1
        slept += w.stats()["sleeping_count"] >= 16
        merged += gi[17] == gi[19]  # the lower stack and the falling stack share an island
    assert compared >= 50 and slept >= 20 and merged >= 5, (compared, slept, merged)
    assert w.stats()["error_flags"] == 0


def test_front_end_skipped_while_everything_sleeps_keeps_its_outputs():
    """Once every body sleeps nothing is integrated, so the front end (Morton codes, sort, tree,
    pairs) is skipped and its last outputs stand.  They must equal what a fresh world computes
    from the same poses, and a pose write must bring the front end back."""
    sc = resting_scene()
    p = bb.make_params(solver=bb.SOLVER_PGS_SOFT, quirks=bb.QUIRKS_PHYSICAL, iterations=8, relax_iterations=8)
    w = bb.world_from_scene(sc, params=p)
    for _ in range(40):
        w.step(DT, 4)
    w.sync()
    assert w.stats()["sleeping_count"] == 18
    keys, ids, pairs = w.debug_read("sorted_keys"), w.debug_read("sorted_ids"), w.debug_read("pairs")
    st = w.read_state()
    sc2 = dict(sc)
    sc2["pos"], sc2["quat"] = st["pos"].copy(), st["quat"].copy()
    sc2["vel"], sc2["omega"] = np.zeros_like(st["vel"]), np.zeros_like(st["omega"])
    fresh = bb.world_from_scene(sc2, params=p)
    fresh.debug_collide(2)
    assert np.array_equal(fresh.debug_read("sorted_keys"), keys)
    assert np.array_equal(fresh.debug_read("sorted_ids"), ids)
    n_pairs = w.stats()["pair_count"]
    assert n_pairs == fresh.stats()["pair_count"] > 0
    assert np.array_equal(fresh.debug_read("pairs")[: 2 * n_pairs], pairs[: 2 * n_pairs])
    # lift one single box far above the others: its ground pair must go
    pos = st["pos"].copy()
    pos[1, 1] += 20.0
    w.write_state(pos=pos)
    w.step(DT, 1)
    w.sync()
    assert w.stats()["pair_count"] == n_pairs - 1
    assert w.stats()["error_flags"] == 0
