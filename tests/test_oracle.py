"""CPU tests of the oracle (the CPU restatement of the reference step).

The reference ships no tests, fixtures or golden vectors, so the oracle's numeric parity with
the reference is unpinned.  What the reference does pin is checked here:
  * its in-shader invariants (coloring.slang:216-292 validator, avbd.slang:915-981 validator,
    the permutation checksum RB_sim.slang:1677-1680),
  * the known-answer demo scenes: scene_3 box towers stay upright
    (src/scene_manager.hpp:327-353) and scene_4's Coulomb outcome on a ramp, sliding iff
    mu < tan(theta) (src/scene_manager.hpp:355-470),
plus hand-computed values of the integer helpers and geometric properties of the collision
routines.
"""
import math

import numpy as np
import pytest

from beatbox import scenes


def test_expand_bits_and_morton_known_values(oracle_lib):
    po = oracle_lib
    wmin, wext = [-64.0] * 3, [128.0] * 3
    # origin -> (64*8 = 512 per axis) -> interleave of 512 = bit 9 on each axis
    code = po.morton([0.0, 0.0, 0.0], wmin, wext)
    assert code == (1 << 29) | (1 << 28) | (1 << 27)
    # below the box clamps to 0, above clamps to 1023 on every axis
    assert po.morton([-100.0, -100.0, -100.0], wmin, wext) == 0
    assert po.morton([100.0, 100.0, 100.0], wmin, wext) == (1 << 30) - 1
    # x only: x cell 1 -> bit 2 (xx*4)
    assert po.morton([-64.0 + 0.125, -64.0, -64.0], wmin, wext) == 4


def test_leaf_aabb_axis_aligned_and_rotated(oracle_lib):
    po = oracle_lib
    a = po.leaf_aabb(0, [0.5, 1.0, 2.0], [1.0, 2.0, 3.0], [0, 0, 0, 1])
    assert np.allclose(a, [0.5, 1.0, 1.0, 1.5, 3.0, 5.0])
    s = math.sin(math.pi / 8)
    c = math.cos(math.pi / 8)  # 45 degrees about y
    a = po.leaf_aabb(0, [0.5, 0.5, 0.5], [0, 0, 0], [0, s, 0, c])
    assert np.allclose(a[[0, 3]], [-math.sqrt(0.5), math.sqrt(0.5)], atol=1e-6)
    a = po.leaf_aabb(1, [0.3, 0.3, 0.3], [1, 1, 1], [0, 0, 0, 1])
    assert np.allclose(a, [0.7, 0.7, 0.7, 1.3, 1.3, 1.3])


def test_box_resting_on_ground_four_contacts(oracle_lib):
    po = oracle_lib
    n, normal, key, pos, dep = po.collide_pair(0, [50, 50, 50], [0, -50, 0], [0, 0, 0, 1],
                                               0, [0.5, 0.5, 0.5], [0, 0.49, 0], [0, 0, 0, 1])
    assert n == 4
    assert np.allclose(normal, [0, 1, 0])
    assert np.allclose(dep, -0.01, atol=1e-9)
    assert np.allclose(np.sort(pos[:, 0]), [-0.5, -0.5, 0.5, 0.5])
    # separated
    assert po.collide_pair(0, [50, 50, 50], [0, -50, 0], [0, 0, 0, 1], 0, [0.5] * 3, [0, 0.6, 0], [0, 0, 0, 1])[0] == 0


def test_sphere_contacts(oracle_lib):
    po = oracle_lib
    n, normal, key, pos, dep = po.collide_pair(1, [0.5] * 3, [0, 0, 0], [0, 0, 0, 1], 1, [0.5] * 3, [0.9, 0, 0],
                                               [0, 0, 0, 1])
    assert n == 1 and key == 20
    assert np.allclose(normal, [1, 0, 0]) and np.isclose(dep[0], -0.1)
    assert np.allclose(pos[0], [0.45, 0, 0])
    # sphere resting on a box face: normal box -> sphere (A = box)
    n, normal, key, pos, dep = po.collide_pair(0, [1, 1, 1], [0, 0, 0], [0, 0, 0, 1], 1, [0.5] * 3, [0, 1.45, 0],
                                               [0, 0, 0, 1])
    assert n == 1 and key == 21 and np.allclose(normal, [0, 1, 0]) and np.isclose(dep[0], -0.05)
    # same pair with the sphere as A flips the normal
    n, normal, key, pos, dep = po.collide_pair(1, [0.5] * 3, [0, 1.45, 0], [0, 0, 0, 1], 0, [1, 1, 1], [0, 0, 0],
                                               [0, 0, 0, 1])
    assert n == 1 and key == 22 and np.allclose(normal, [0, -1, 0])
    # sphere centre inside the box: deepest face is +y
    n, normal, key, pos, dep = po.collide_pair(0, [1, 1, 1], [0, 0, 0], [0, 0, 0, 1], 1, [0.25] * 3, [0, 0.9, 0],
                                               [0, 0, 0, 1])
    assert n == 1 and np.allclose(normal, [0, 1, 0]) and np.isclose(dep[0], -0.1 - 0.25)


def test_sat_frame_quirk_only_matters_for_general_rotations(oracle_lib):
    """C = R_A R_B^T (reference) equals the consistent frame when either box is axis aligned."""
    po = oracle_lib
    q = scenes.random_rotations(7, 0, 400)
    rng = np.random.default_rng(0)
    differ = 0
    for k in range(200):
        pb = rng.uniform(-1.2, 1.2, 3)
        h = [0.5, 0.5, 0.5]
        ref = po.collide_pair(0, h, [0, 0, 0], [0, 0, 0, 1], 0, h, pb, q[k], True)[0]
        fix = po.collide_pair(0, h, [0, 0, 0], [0, 0, 0, 1], 0, h, pb, q[k], False)[0]
        assert ref == fix
        ref = po.collide_pair(0, h, [0, 0, 0], q[2 * k], 0, h, pb, q[2 * k + 1], True)[0] > 0
        fix = po.collide_pair(0, h, [0, 0, 0], q[2 * k], 0, h, pb, q[2 * k + 1], False)[0] > 0
        differ += ref != fix
    assert differ > 0  # the reference's relative rotation is not the consistent one in general


def _oracle(po, sc, **kw):
    p = po.default_params()
    for k, v in kw.items():
        setattr(p, k, v)
    if sc.get("bounds") is not None:
        p.world_min[:] = sc["bounds"][0]
        p.world_extent[:] = sc["bounds"][1]
    return po.Oracle(sc, params=p)


def test_front_end_invariants_and_pairs_vs_brute_force(oracle_lib):
    po = oracle_lib
    sc = scenes.mixed_column(n_bodies=600, seed=3)
    o = _oracle(po, sc)
    o.collide(1)
    n = sc["n"]
    cnt, b = o.debug_read(3)
    ids = b[: 4 * cnt].view(np.uint32)
    assert cnt == n and sorted(ids.tolist()) == list(range(n))  # permutation (RB_sim.slang:1677-1680)
    cnt, b = o.debug_read(2)
    keys = b[: 4 * cnt].view(np.uint32)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    # LBVH: every node reachable exactly once from the root, leaves cover 0..n-1 in order
    cnt, b = o.debug_read(4)
    child = b[: 4 * cnt].view(np.int32).reshape(-1, 2)
    seen, leaves, stack = set(), [], [0]
    while stack:
        nd = stack.pop()
        assert nd not in seen
        seen.add(nd)
        if nd >= n - 1:
            leaves.append(nd - (n - 1))
        else:
            stack.extend([child[nd, 1], child[nd, 0]])
    assert leaves == list(range(n))
    # pair set == brute-force closed-interval overlap of the leaf boxes
    cnt, b = o.debug_read(5)
    box = b[: 4 * cnt].view(np.float32).reshape(-1, 6)
    mn, mx = box[:, :3], box[:, 3:]
    ov = np.all((mn[:, None, :] <= mx[None, :, :]) & (mx[:, None, :] >= mn[None, :, :]), axis=2)
    ii, jj = np.nonzero(np.triu(ov, 1))
    cnt, b = o.debug_read(7)
    pairs = b[: 4 * cnt].view(np.uint32).reshape(-1, 2)
    assert np.array_equal(pairs, np.stack([ii, jj], 1))


def test_colourings_are_valid(oracle_lib):
    po = oracle_lib
    sc = scenes.box_grid(n_side=5, layers=4)
    for solver in (1, 2):
        o = _oracle(po, sc, solver=solver, quirks=0, iterations=4, relax_iterations=4, avbd_iterations=2)
        for _ in range(40):
            o.step(1 / 60, 2)
        st = o.stats()
        assert st["graph_color_violations"] == 0 and st["graph_color_overflow"] == 0
        assert st["manifold_count"] > 0
        if solver == 2:
            assert st["avbd_violations"] == 0 and st["avbd_color_count"] > 0


def test_thread_count_does_not_change_results(oracle_lib):
    po = oracle_lib
    sc = scenes.box_grid(n_side=5, layers=3)
    outs = []
    for threads in (1, 4):
        for solver in (1, 2):
            o = po.Oracle(sc, threads=threads)
            p = po.default_params()
            p.solver, p.quirks = solver, 0
            o.set_params(p)
            for _ in range(30):
                o.step(1 / 60, 2)
            outs.append(o.state()["pos"])
    assert np.array_equal(outs[0], outs[2]) and np.array_equal(outs[1], outs[3])


def _tower(heights, spacing=3.0, inertia="physical", density=5.0):
    sb = scenes.SceneBuilder(inertia)
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    for t, hgt in enumerate(heights):
        pos = [[t * spacing, 0.5 + 1.0 * k, 0.0] for k in range(hgt)]
        sb.add(pos, [[0, 0, 0, 1]] * hgt, [[0.5] * 3] * hgt, 0, scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY,
               density)
    return sb.build()


@pytest.mark.parametrize("solver", [1, 2])
def test_scene3_towers_stay_upright(oracle_lib, solver):
    """scene_3 (src/scene_manager.hpp:327-353): towers of 5 / 8 / 12 cubes must stay upright."""
    sc = _tower([5, 8, 12])
    o = _oracle(oracle_lib, sc, solver=solver, quirks=0, iterations=8, relax_iterations=8)
    for _ in range(240):
        o.step(1 / 60, 2)
    pos = o.state()["pos"][1:]
    x0 = np.concatenate([np.full(h, 3.0 * t) for t, h in enumerate([5, 8, 12])])
    assert np.abs(pos[:, 0] - x0).max() < 0.05
    assert np.abs(pos[:, 2]).max() < 0.05
    top = np.cumsum([5, 8, 12]) - 1
    assert np.all(pos[top, 1] > np.array([5, 8, 12]) - 0.7)


def _ramp(theta_deg, mu, solver):
    th = math.radians(theta_deg)
    q = [0, 0, math.sin(th / 2), math.cos(th / 2)]  # rotate about z
    sb = scenes.SceneBuilder("physical")
    sb.add([[0, 0, 0]], [q], [[6, 0.25, 2]], 0, 0, 0.0, friction=mu)
    # box resting on the ramp's upper face
    nrm = np.array([-math.sin(th), math.cos(th), 0.0])
    c = nrm * (0.25 + 0.5 + 0.002)
    sb.add([c], [q], [[0.5] * 3], 0, scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 5.0, friction=mu)
    return sb.build(), np.array([math.cos(th), math.sin(th), 0.0])


@pytest.mark.parametrize("theta,mu", [(15, 0.5), (15, 1.0), (30, 0.2), (30, 1.0)])
def test_scene4_coulomb_outcome(oracle_lib, theta, mu):
    """scene_4 (src/scene_manager.hpp:355-470): a box on a ramp slides iff mu < tan(theta)."""
    sc, down = _ramp(theta, mu, 1)
    o = _oracle(oracle_lib, sc, solver=1, quirks=0, iterations=8, relax_iterations=8)
    p0 = o.state()["pos"][1].copy()
    for _ in range(90):
        o.step(1 / 60, 2)
    disp = o.state()["pos"][1] - p0
    slid = -np.dot(disp, down)  # distance travelled down the slope
    if mu < math.tan(math.radians(theta)):
        assert slid > 0.3
    else:
        assert abs(slid) < 0.05


@pytest.mark.parametrize("solver", [1, 2])
@pytest.mark.parametrize("scene", ["boxes", "voxels"])
def test_frozen_pairs_carry_over_gives_the_recomputed_result(oracle_lib, solver, scene):
    """Pairs whose bodies were asleep (or static) at the last narrow phase and still are keep
    their manifolds instead of recomputing them; on piles that fall asleep this gives the same
    bits as recomputing every pair (states and contacts)."""
    import beatbox as bb

    sc = scenes.box_grid(n_side=4, layers=2) if scene == "boxes" else scenes.voxel_pile(9, seed=2)
    out = []
    for carry in (True, False):
        p = oracle_lib.default_params()
        p.quirks = 0
        p.solver = solver
        p.iterations = p.relax_iterations = 8
        p.avbd_iterations = 4
        o = oracle_lib.Oracle(sc, params=p, threads=4)
        o.set_carry_frozen(carry)
        for _ in range(300):
            o.step(1.0 / 60.0, 4)
        cnt, buf = o.debug_read(9)
        out.append((o.state(), buf[: cnt * bb.CONTACT_DTYPE.itemsize].copy(), o.stats()["sleeping_count"]))
    (a, ca, sa), (b, cb, sb) = out
    assert sa > 0 and sa == sb
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(ca, cb)
