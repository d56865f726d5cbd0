"""GPU tests of voxel (concave) bodies through the C ABI, against the oracle.

Tolerances (as for the other shapes): front end bit-exact (leaf boxes of the off-centre voxel
grid boxes, tree, pairs); manifold identities bit-exact (bodies, face key 90..95, contact count,
sampled-voxel feature ids); normals 1e-5, contact points and depths 1e-4 m against the FP64
oracle; one step from a contact-rich state 1e-4 of the world's scale on positions.
"""
import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
FLAGS = scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY


def mixed_voxel_scene(seed=3):
    """Voxel pile with boxes and spheres among the voxel bodies (voxel-box, voxel-sphere and
    voxel-voxel pairs, plus the ordinary shapes)."""
    sc = scenes.voxel_pile(36, seed=seed)
    sb = scenes.SceneBuilder()
    sb.parts = []
    sb.voxel_shapes = []
    gx, gz = np.arange(12) % 4, np.arange(12) // 4
    pos = np.stack([-2.4 + 1.6 * gx, np.full(12, 6.5), -1.6 + 1.6 * gz], 1) + scenes.uniform(seed, 50, 36, -0.1, 0.1).reshape(12, 3)
    sb.add(pos[:6], scenes.random_rotations(seed, 60, 6), np.full((6, 3), 0.25), scenes.SHAPE_BOX, FLAGS, 60.0)
    sb.add(pos[6:], np.tile([0, 0, 0, 1.0], (6, 1)), np.full((6, 3), 0.2), scenes.SHAPE_SPHERE, FLAGS, 30.0)
    extra = {k: np.concatenate([p[k] for p in sb.parts]) for k in sb.parts[0]}
    out = {k: np.ascontiguousarray(np.concatenate([sc[k], extra[k]])) for k in extra}
    out["n"] = out["pos"].shape[0]
    out["bounds"] = None
    out["voxel_shapes"] = sc["voxel_shapes"]
    return out


def params_for(po, sc, **kw):
    p = po.default_params()
    p.quirks = bb.QUIRKS_PHYSICAL
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def oread(o, code, dtype=None):
    cnt, buf = o.debug_read(code)
    if code == 8:
        return buf[: cnt * bb.MANIFOLD_DTYPE.itemsize].view(bb.MANIFOLD_DTYPE)
    if code == 9:
        return buf[: cnt * bb.CONTACT_DTYPE.itemsize].view(bb.CONTACT_DTYPE)
    return buf[: cnt * np.dtype(dtype).itemsize].view(dtype)


def settled(po, sc, p, steps):
    o = po.Oracle(sc, params=p, threads=4)
    for _ in range(steps):
        o.step(DT, 4)
    st = o.state()
    sc2 = dict(sc)
    for k, a in (("pos", "pos"), ("quat", "quat"), ("vel", "vel"), ("omega", "omega")):
        sc2[k] = st[a].astype(np.float32)
    return sc2


def test_voxel_front_end_bit_exact(oracle_lib):
    sc = mixed_voxel_scene()
    p = params_for(oracle_lib, sc)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_lib.Oracle(sc, params=p)
    w.debug_collide(1)
    o.collide(1)
    assert np.array_equal(w.debug_read("sorted_ids"), oread(o, 3, np.uint32))
    assert np.array_equal(w.debug_read("leaf_aabb"), oread(o, 5, np.float32))
    assert np.array_equal(w.debug_read("node_aabb"), oread(o, 6, np.float32))
    assert np.array_equal(w.debug_read("pairs"), oread(o, 7, np.uint32))


@pytest.mark.parametrize("steps", [45, 90])
def test_voxel_narrow_phase_matches_oracle(oracle_lib, steps):
    base = mixed_voxel_scene()
    p = params_for(oracle_lib, base, solver=bb.SOLVER_AVBD, avbd_iterations=4)
    sc = settled(oracle_lib, base, p, steps)
    w = bb.world_from_scene(sc, params=p)
    o = oracle_lib.Oracle(sc, params=p)
    w.debug_collide(2)
    o.collide(2)
    gm, rm = w.debug_read("manifolds"), oread(o, 8)
    assert len(gm) == len(rm) and (gm["key"] >= 90).sum() > 10
    for f in ("body_a", "body_b", "key", "contact_count"):
        assert np.array_equal(gm[f], rm[f]), f
    assert np.abs(gm["normal"] - rm["normal"]).max() < 1e-5
    gc, rc = w.debug_read("contacts"), oread(o, 9)
    mask = (np.arange(8)[None, :] < gm["contact_count"][:, None]).ravel()
    assert np.abs(gc["position"][mask] - rc["position"][mask]).max() < 1e-4
    assert np.abs(gc["penetration"][mask] - rc["penetration"][mask]).max() < 1e-4
    assert np.array_equal(gc["feature"][mask], rc["feature"][mask])


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
def test_voxel_one_step_within_tolerance(oracle_lib, solver):
    base = mixed_voxel_scene()
    p = params_for(oracle_lib, base, solver=solver, iterations=8, relax_iterations=8, avbd_iterations=4)
    sc = settled(oracle_lib, base, p, 45)
    sc["flags"] = base["flags"].copy()  # everyone awake
    w = bb.world_from_scene(sc, params=p)
    o = oracle_lib.Oracle(sc, params=p)
    o.step(DT, 4)
    w.step(DT, 4)
    w.sync()
    assert w.stats()["manifold_count"] > 30
    g, r = w.read_state(), o.state()
    dyn = (sc["flags"] & bb.BODY_DYNAMIC) != 0
    perr = np.abs(g["pos"][dyn] - r["pos"][dyn]).max() / np.abs(r["pos"][dyn]).max()
    verr = np.abs(g["vel"][dyn] - r["vel"][dyn]).max()
    assert perr < 1e-4, perr
    assert verr < 2e-4 * max(np.abs(r["vel"][dyn]).max(), 1.0), verr


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
def test_voxel_pile_settles_on_gpu(solver):
    sc = scenes.voxel_pile(24, seed=1)
    p = bb.make_params(solver=solver, quirks=bb.QUIRKS_PHYSICAL, iterations=8, relax_iterations=8, avbd_iterations=4)
    w = bb.world_from_scene(sc, params=p)
    for _ in range(300):
        w.step(DT, 4)
    st, x = w.stats(), w.read_state()
    assert x["pos"][1:, 1].min() > 0.05
    assert np.abs(x["vel"][1:]).max() < 0.2
    assert st["sleeping_count"] >= 0.7 * 24  # chaotic: the FP32 trajectory is not the oracle's
    assert st["error_flags"] == 0


def test_voxel_steps_are_deterministic():
    sc = mixed_voxel_scene(seed=4)
    outs = []
    for _ in range(2):
        w = bb.world_from_scene(sc, params=bb.make_params(solver=bb.SOLVER_PGS_SOFT, quirks=bb.QUIRKS_PHYSICAL))
        for _ in range(60):
            w.step(DT, 4)
        outs.append(w.read_state())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k])


def test_voxel_shape_inertia_from_the_shape_matches_scene():
    """A voxel body added without explicit inertia gets the same mass and inverse inertia as the
    scene builder computes from the shape's unit values."""
    sc = scenes.voxel_pile(3, seed=0)
    w = bb.World(8)
    h = w.add_voxel_shape(sc["voxel_shapes"][0]["solid"], sc["voxel_shapes"][0]["voxel_size"])
    d = bb.BodyDesc()
    d.position[:] = [0, 1, 0]
    d.rotation[:] = [0, 0, 0, 1]
    d.shape = h
    d.flags = FLAGS
    d.density = 1000.0
    d.inertia_mode = bb.INERTIA_PHYSICAL
    w.add_bodies([d])
    a = w.debug_read("body_inertia")
    k = int(np.nonzero((sc["shape"] == scenes.SHAPE_VOXEL) & (sc["voxel"] == 0))[0][0])
    assert np.array_equal(a[0, :3], sc["inv_inertia"][k]) and np.array_equal(a[0, 3:6], sc["inv_inertia_off"][k])


def test_voxel_worlds_are_the_same_alone_and_in_a_batch():
    """Two voxel piles stepped as independent worlds of one batch give the bits of each pile
    stepped alone (six-slot voxel pairs, world-local colouring, world-prefixed sort)."""
    a, b = scenes.voxel_pile(12, seed=5), scenes.voxel_pile(15, seed=6)
    p = bb.make_params(solver=bb.SOLVER_PGS_SOFT, quirks=bb.QUIRKS_PHYSICAL)
    alone = []
    for sc in (a, b):
        w = bb.World(sc["n"], pairs_per_body=64)
        w.add_world(sc, sc["bounds"][0], sc["bounds"][1])
        w.set_params(p)
        for _ in range(40):
            w.step(DT, 4)
        alone.append(w.read_state())
    w = bb.World(a["n"] + b["n"], pairs_per_body=64)
    w.add_world(a, a["bounds"][0], a["bounds"][1])
    w.add_world(b, b["bounds"][0], b["bounds"][1])
    w.set_params(p)
    for _ in range(40):
        w.step(DT, 4)
    both = w.read_state()
    assert w.stats()["error_flags"] == 0
    for k in both:
        assert np.array_equal(both[k][: a["n"]], alone[0][k]), k
        assert np.array_equal(both[k][a["n"]:], alone[1][k]), k
