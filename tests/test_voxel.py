"""CPU tests of voxel (concave) bodies: the library's host shape build and the oracle's voxel
narrow phase (collision_detection.slang:1001-1512, build_voxel_shape scene_manager.hpp:488-560).

The reference has no tests for this path either.  Pinned here:
  * the shape build against hand-computed values (a solid block's centre of mass, surface count
    and exact box inertia; the L's centre of mass and its product of inertia) and against the
    oracle's own restatement of the builder (origin, box, surface list);
  * the narrow phase against a hand-computed resting contact (a voxel cube 1 cm into the
    ground: one manifold on the ground's +y face, the four corner cells at depth 1 cm);
  * the contact identities a resting pair keeps from step to step (warm start);
  * settling of a voxel pile under both solvers without tunnelling.
"""
import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

DT = 1.0 / 60.0


def cell_inertia(solid, vs):
    """Independent restatement: centre of mass and inertia of unit-density cubes."""
    z, y, x = np.nonzero(solid)
    c = (np.stack([x, y, z], 1) + 0.5) * vs
    com = c.mean(0)
    r = c - com
    m = vs ** 3
    inertia = np.zeros((3, 3))
    for v in r:
        inertia += m * (np.dot(v, v) * np.eye(3) - np.outer(v, v))
    inertia += len(r) * m * vs * vs / 6.0 * np.eye(3)
    return com, inertia


@pytest.mark.parametrize("shape", ["block", "l", "cross", "frame"])
def test_voxel_shape_build_known_values(shape):
    vs = 0.2
    g = {"block": np.ones((3, 3, 3), np.uint8), "l": scenes.voxel_l_shape(), "cross": scenes.voxel_cross(),
         "frame": scenes.voxel_frame()}[shape]
    info = bb.voxel_shape_info(g, vs)
    com, inertia = cell_inertia(g, vs)
    assert info["solid_count"] == int(g.sum())
    assert np.allclose(info["grid_origin"], -com, atol=1e-6)
    assert np.allclose(info["box_min"], -com, atol=1e-6)
    assert np.allclose(info["box_max"], -com + np.array(g.shape[::-1]) * vs, atol=1e-6)
    assert np.isclose(info["unit_mass"], g.sum() * vs ** 3, rtol=1e-6)
    inv = np.linalg.inv(inertia)
    ui = info["unit_inv_inertia"]
    full = np.array([[ui[0], ui[3], ui[4]], [ui[3], ui[1], ui[5]], [ui[4], ui[5], ui[2]]])
    assert np.allclose(full, inv, rtol=1e-5, atol=1e-6 * np.abs(inv).max())
    if shape == "block":
        # a solid 3x3x3 block: one interior cell; the exact box inertia m (a^2 + b^2) / 12
        assert info["surface_count"] == 26
        side = 3 * vs
        assert np.allclose(np.diag(inertia), 27 * vs ** 3 * 2 * side * side / 12.0)
    if shape == "l":
        assert abs(ui[3]) > 1e-3 * ui[0]  # the L has a product of inertia in its plane


def test_surface_list_order_and_directions():
    g = np.ones((1, 1, 3), np.uint8)  # three cells along x
    info = bb.voxel_shape_info(g, 1.0)
    s = info["surface"]
    assert info["surface_count"] == 3
    cells = [(int(e) & 0xFF, (int(e) >> 8) & 0xFF, (int(e) >> 16) & 0xFF, int(e) >> 24) for e in s]
    # z, y, x order; first empty neighbour in -x, +x, -y, +y, -z, +z order
    assert cells == [(0, 0, 0, 0), (1, 0, 0, 2), (2, 0, 0, 1)]


def test_bad_voxel_grids_rejected():
    with pytest.raises(bb.BeatboxError):
        bb.voxel_shape_info(np.zeros((2, 2, 2), np.uint8), 0.1)
    with pytest.raises(bb.BeatboxError):
        bb.voxel_shape_info(np.ones((2, 2, 2), np.uint8), 0.0)


def test_oracle_builder_matches_library(oracle_lib):
    sc = scenes.voxel_pile(6)
    o = oracle_lib.Oracle(sc)
    for k, v in enumerate(sc["voxel_shapes"]):
        lib = bb.voxel_shape_info(v["solid"], v["voxel_size"])
        orc = oracle_lib.voxel_shape(o, k)
        for key in ("grid_origin", "box_min", "box_max"):
            assert np.array_equal(lib[key], orc[key])
        assert lib["solid_count"] == orc["solid_count"] and lib["surface_count"] == orc["surface_count"]
        assert np.array_equal(lib["surface"], orc["surface"])


def cube_on_ground(depth, vs=0.2, yaw=0.0):
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    k = sb.add_voxel_shape(np.ones((3, 3, 3), np.uint8), vs)
    h = 0.5 * yaw
    sb.add_voxel([[0.0, 1.5 * vs - depth, 0.0]], [[0, np.sin(h), 0, np.cos(h)]], k, scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY)
    return sb.build()


def oread(o, code):
    cnt, buf = o.debug_read(code)
    dt = bb.MANIFOLD_DTYPE if code == 8 else bb.CONTACT_DTYPE
    return buf[: cnt * dt.itemsize].view(dt)


def test_voxel_cube_resting_contact_known_answer(oracle_lib):
    sc = cube_on_ground(0.01)
    o = oracle_lib.Oracle(sc, params=oracle_lib.default_params())
    o.collide(2)
    m = oread(o, 8)
    assert len(m) == 1  # only the ground's +y face (code 3) sees the cube
    assert m["key"][0] == 93 and m["contact_count"][0] == 4
    assert np.allclose(np.abs(m["normal"][0]), [0, 1, 0], atol=1e-12)
    c = oread(o, 9)[:4]
    # the four bottom corner cells' centres, 1 cm deep
    pts = sorted(map(tuple, np.round(c["position"], 6)))
    assert pts == sorted([(x, 0.09, z) for x in (-0.2, 0.2) for z in (-0.2, 0.2)])
    assert np.allclose(c["penetration"], -0.01, atol=1e-6)
    # feature ids: the sampled cell (x | y << 8 | z << 16), corner index 0 (one point per cell)
    cells = sorted((int(f) & 0xFF, (int(f) >> 8) & 0xFF, (int(f) >> 16) & 0xFF) for f in c["feature"])
    assert cells == [(0, 0, 0), (0, 0, 2), (2, 0, 0), (2, 0, 2)]


def test_voxel_cube_touching_and_separated(oracle_lib):
    # exactly touching: a manifold at depth 0 (the margin band keeps resting contacts alive)
    o = oracle_lib.Oracle(cube_on_ground(0.0), params=oracle_lib.default_params())
    o.collide(2)
    c = oread(o, 9)
    assert len(oread(o, 8)) == 1 and np.allclose(c["penetration"][:4], 0.0, atol=1e-6)
    # 1 cm above: a sample centre more than its support radius outside the face is no contact
    o = oracle_lib.Oracle(cube_on_ground(-0.01), params=oracle_lib.default_params())
    o.collide(2)
    assert len(oread(o, 8)) == 0


def test_voxel_pair_emits_one_manifold_per_face(oracle_lib):
    # an L lying flat on top of a block: the L's cells touch the block's +y face only
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    kb = sb.add_voxel_shape(np.ones((2, 4, 4), np.uint8), 0.2)  # 0.8 x 0.8 x 0.4 block
    kl = sb.add_voxel_shape(scenes.voxel_l_shape(), 0.2)
    flat = [np.sin(-np.pi / 4), 0, 0, np.cos(-np.pi / 4)]  # L plane (x, y) -> (x, z)
    sb.add_voxel([[0, 0.4 - 0.005, 0]], [[0, 0, 0, 1]], kb, scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY)
    sb.add_voxel([[0.0, 0.8 + 0.2 - 0.01, 0.0]], [flat], kl, scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY)
    o = oracle_lib.Oracle(sb.build(), params=oracle_lib.default_params())
    o.collide(2)
    m = oread(o, 8)
    keys = sorted(int(k) for k, a, b in zip(m["key"], m["body_a"], m["body_b"]) if {int(a), int(b)} == {1, 2})
    assert keys and all(90 <= k <= 95 for k in keys)
    assert len(keys) == len(set(keys))


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
def test_voxel_pile_settles_without_tunnelling(oracle_lib, solver):
    sc = scenes.voxel_pile(24, seed=1)
    p = oracle_lib.default_params()
    p.solver = solver
    p.quirks = bb.QUIRKS_PHYSICAL
    p.iterations = p.relax_iterations = 8
    p.avbd_iterations = 4
    o = oracle_lib.Oracle(sc, threads=4, params=p)
    for _ in range(300):
        o.step(DT, 4)
    st, x = o.stats(), o.state()
    assert x["pos"][1:, 1].min() > 0.05  # nothing sank through the ground (top at y = 0)
    assert np.abs(x["vel"][1:]).max() < 0.2
    assert st["sleeping_count"] >= 0.8 * 24
    assert st["max_penetration"] < 0.12


def test_voxel_resting_contacts_keep_their_identity(oracle_lib):
    sc = cube_on_ground(0.005)
    p = oracle_lib.default_params()
    p.quirks = bb.QUIRKS_PHYSICAL
    p.solver = bb.SOLVER_PGS_SOFT
    p.flags &= ~(1 << 7)  # sleeping off: keep the pair active
    o = oracle_lib.Oracle(sc, params=p)
    for _ in range(40):  # past the transient of the initial 5 mm overlap
        o.step(DT, 4)
    w0 = oread(o, 9)["warm_start"][:4].copy()
    for _ in range(5):
        o.step(DT, 4)
        assert o.stats()["fresh_contacts"] == 0
    # every contact inherited its impulses in each of the 20 substeps
    assert np.array_equal(oread(o, 9)["warm_start"][:4], np.minimum(w0 + 20, 255))


def test_served_worlds_take_boxes_and_spheres_only():
    with pytest.raises(ValueError):
        bb.scene_request_arrays(scenes.voxel_pile(3))
