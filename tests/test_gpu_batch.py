"""GPU tests of the batched-worlds mode and of the two PGS schedules.

Both are pure reorganisations of the same arithmetic, so the bar is bitwise equality:
  * a world stepped inside a batch equals the same world stepped alone (its body ids are
    shifted by the world's first id; every hash, sort and traversal works on world-local
    ids and per-world ranges);
  * the dataflow PGS schedule (per-body sequence counters) equals the colour-barrier
    schedule (grid barrier between colours), since every body still sees its constraints
    in colour order.
"""
import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def scene_bounds(sc, margin=4.0):
    if sc.get("bounds") is not None:
        return sc["bounds"]
    lo = sc["pos"].min(axis=0) - margin
    hi = sc["pos"].max(axis=0) + margin
    return lo.tolist(), np.maximum(hi - lo, 1.0).tolist()


def small_column(seed):
    return scenes.mixed_column(n_bodies=400, seed=seed)


def tiny_stack():
    sb = scenes.SceneBuilder()
    sb.add_static_box([0, -50, 0], [50, 50, 50])
    sb.add([[0, 0.5 + 1.0 * k, 0] for k in range(5)], [[0, 0, 0, 1]] * 5, [[0.5] * 3] * 5, 0,
           scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY, 1.0)
    return sb.build()


WORLDS = [
    lambda: scenes.box_grid(n_side=5, layers=3),
    lambda: small_column(3),
    tiny_stack,
    lambda: scenes.pyramids(n_pyramids=2, boxes_per=55, gap=-0.002),
    lambda: small_column(4),
]


def params(solver, **kw):
    p = bb.make_params(solver=solver, quirks=bb.QUIRKS_PHYSICAL, **kw)
    if solver == bb.SOLVER_AVBD:
        p.avbd_iterations = 4
    return p


def run_batch(scs, p, steps, substeps):
    total = sum(int(s["n"]) for s in scs)
    w = bb.World(total)
    firsts = []
    for k, sc in enumerate(scs):
        lo, ext = scene_bounds(sc)
        wi, first = w.add_world(sc, lo, ext)
        assert wi == k
        firsts.append(first)
    assert w.n_worlds == len(scs)
    w.set_params(p)
    for _ in range(steps):
        w.step(DT, substeps)
    st = w.read_state()
    stats = w.stats()
    w.close()
    return [{k: v[f:f + int(sc["n"])] for k, v in st.items()} for f, sc in zip(firsts, scs)], stats


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
def test_batched_world_equals_world_alone(solver):
    scs = [f() for f in WORLDS]
    p = params(solver)
    batch, stats = run_batch(scs, p, steps=30, substeps=2)
    assert stats["error_flags"] == 0
    for k, sc in enumerate(scs):
        alone, _ = run_batch([sc], p, steps=30, substeps=2)
        for key in alone[0]:
            assert np.array_equal(batch[k][key], alone[0][key]), (k, key)


def test_overlapping_worlds_never_interact():
    """Three copies of one scene occupying the same space: with no cross-world pairs every
    copy evolves exactly like the scene alone."""
    sc = small_column(5)
    p = params(bb.SOLVER_PGS_SOFT)
    batch, _ = run_batch([sc, sc, sc], p, steps=40, substeps=2)
    alone, _ = run_batch([sc], p, steps=40, substeps=2)
    for k in range(3):
        for key in alone[0]:
            assert np.array_equal(batch[k][key], alone[0][key]), (k, key)


def test_batched_pairs_stay_inside_worlds():
    scs = [small_column(6), small_column(6)]
    total = sum(int(s["n"]) for s in scs)
    w = bb.World(total)
    for sc in scs:
        w.add_world(sc, *scene_bounds(sc))
    w.set_params(params(bb.SOLVER_PGS_SOFT))
    for _ in range(20):
        w.step(DT, 1)
    w.debug_collide(2)
    man = w.debug_read("manifolds")
    n0 = int(scs[0]["n"])
    assert len(man) > 0
    wa = man["body_a"] >= n0
    wb = man["body_b"] >= n0
    assert np.array_equal(wa, wb)
    assert 0 < wa.sum() < len(man)


def test_mixing_plain_and_batched_is_rejected():
    sc = tiny_stack()
    w = bb.World(64)
    w.add_world(sc, *scene_bounds(sc))
    with pytest.raises(bb.BeatboxError):
        w.add_scene(sc)
    w.close()
    w = bb.World(64)
    w.add_scene(sc)
    with pytest.raises(bb.BeatboxError):
        w.add_world(sc, *scene_bounds(sc))
    w.close()


@pytest.mark.parametrize("name", ["mixed_3000", "pyramids_4x300"])
def test_dataflow_schedule_equals_colour_barrier(name):
    sc = (scenes.mixed_column(n_bodies=3000, seed=2) if name == "mixed_3000"
          else scenes.pyramids(n_pyramids=4, boxes_per=300, gap=-0.002))
    outs = []
    for schedule in (bb.SCHEDULE_DATAFLOW, bb.SCHEDULE_COLOUR_BARRIER):
        p = params(bb.SOLVER_PGS_SOFT, schedule=schedule)
        w = bb.world_from_scene(sc, params=p)
        for _ in range(40):
            w.step(DT, 4)
        outs.append(w.read_state())
        assert w.stats()["error_flags"] == 0
        w.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.parametrize("name", ["mixed_3000", "pyramids_200x1000"])
def test_staging_the_next_item_equals_loading_it(name):
    """The colour-barrier kernel that stages each thread's next item of a colour in shared memory
    while the current one computes runs the same arithmetic on the same data.  In the 200k-box
    pyramids (over 400k manifolds in about a dozen colours, on at most 148 x 256 threads) the
    threads run several items of the largest colours, so the staged path carries them."""
    big = name == "pyramids_200x1000"
    sc = scenes.pyramids(n_pyramids=200, boxes_per=1000, seed=0) if big else scenes.mixed_column(n_bodies=3000, seed=2)
    outs = []
    for stage in (0, 1):
        p = params(bb.SOLVER_PGS_SOFT, schedule=bb.SCHEDULE_COLOUR_BARRIER, pgs_stage_next=stage)
        w = bb.world_from_scene(sc, params=p)
        for _ in range(4 if big else 40):
            w.step(DT, 4)
        outs.append(w.read_state())
        st = w.stats()
        assert st["error_flags"] == 0
        if big:
            assert st["manifold_count"] > 400_000  # the largest colours hold more items than the grid has threads
        w.close()
    for o in outs[1:]:
        for k in outs[0]:
            assert np.array_equal(outs[0][k], o[k]), k


def test_world_added_to_a_running_batch_leaves_the_others_unchanged():
    """Serving pattern: world B joins after A has run 10 steps; A continues exactly as alone
    (its warm-start contacts and sort order survive the join) and B runs as if alone."""
    a, b = small_column(7), tiny_stack()
    p = params(bb.SOLVER_PGS_SOFT)
    w = bb.World(int(a["n"]) + int(b["n"]))
    w.add_world(a, *scene_bounds(a))
    w.set_params(p)
    for _ in range(10):
        w.step(DT, 2)
    _, fb = w.add_world(b, *scene_bounds(b))
    for _ in range(10):
        w.step(DT, 2)
    st = w.read_state()
    w.close()
    alone_a, _ = run_batch([a], p, steps=20, substeps=2)
    alone_b, _ = run_batch([b], p, steps=10, substeps=2)
    na = int(a["n"])
    for key in st:
        assert np.array_equal(st[key][:na], alone_a[0][key]), key
        assert np.array_equal(st[key][fb:fb + int(b["n"])], alone_b[0][key]), key


def test_autotune_keeps_results_bit_identical():
    sc = scenes.mixed_column(n_bodies=2000, seed=3)
    p = params(bb.SOLVER_PGS_SOFT)
    w = bb.world_from_scene(sc, params=p)
    tuned = w.autotune(DT, 2, trial_steps=1)
    steps = w.stats()["substeps_run"] // 2
    assert steps >= 4 and set(tuned) >= {"schedule", "broad_threads", "narrow_blocks_per_sm"}
    for _ in range(5):
        w.step(DT, 2)
    ref = bb.world_from_scene(sc, params=p)
    for _ in range(steps + 5):
        ref.step(DT, 2)
    a, b = w.read_state(), ref.read_state()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def resting_boxes(x0):
    """Four boxes resting on a ground box from the start: they fall asleep after the quiet time."""
    sb = scenes.SceneBuilder()
    sb.add_static_box([x0, -50, 0], [50, 50, 50])
    pos = [[x0 - 2.4 + 1.6 * k, 0.499, 0.0] for k in range(4)]
    sb.add(pos, [[0, 0, 0, 1.0]] * 4, [[0.5] * 3] * 4, scenes.SHAPE_BOX, scenes.BODY_DYNAMIC | scenes.BODY_GRAVITY,
           1000.0)
    return sb.build()


def test_batched_worlds_asleep_keep_their_front_end_outputs():
    """Once every body of every world sleeps, the batched front end (two-digit world-id sort,
    world-bounded traversal) is skipped and its outputs stand: they must equal a fresh batch's
    on the same poses, and a pose written into one world must bring the front end back."""
    scs = [resting_boxes(0.0), resting_boxes(200.0), resting_boxes(400.0)]
    p = params(bb.SOLVER_PGS_SOFT, iterations=8, relax_iterations=8)
    total = sum(int(s["n"]) for s in scs)

    boxes = [scene_bounds(sc, margin=60.0) for sc in scs]  # the same Morton box for both batches

    def batch(worlds):
        w = bb.World(total)
        for sc, box in zip(worlds, boxes):
            w.add_world(sc, *box)
        w.set_params(p)
        return w

    w = batch(scs)
    for _ in range(40):
        w.step(DT, 4)
    w.sync()
    assert w.stats()["sleeping_count"] == 12
    keys, ids, pairs = w.debug_read("sorted_keys"), w.debug_read("sorted_ids"), w.debug_read("pairs")
    n_pairs = w.stats()["pair_count"]
    st = w.read_state()
    rest, first = [], 0
    for sc in scs:
        n = int(sc["n"])
        s2 = dict(sc)
        s2["pos"], s2["quat"] = st["pos"][first:first + n].copy(), st["quat"][first:first + n].copy()
        s2["vel"], s2["omega"] = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
        rest.append(s2)
        first += n
    fresh = batch(rest)
    fresh.debug_collide(2)
    assert np.array_equal(fresh.debug_read("sorted_keys"), keys)
    assert np.array_equal(fresh.debug_read("sorted_ids"), ids)
    assert n_pairs == fresh.stats()["pair_count"] > 0
    assert np.array_equal(fresh.debug_read("pairs")[: 2 * n_pairs], pairs[: 2 * n_pairs])
    # lift one box of the second world far above its ground: its ground pair must go
    pos = st["pos"].copy()
    pos[int(scs[0]["n"]) + 1, 1] += 20.0
    w.write_state(pos=pos)
    w.step(DT, 1)
    w.sync()
    assert w.stats()["pair_count"] == n_pairs - 1
    assert w.stats()["error_flags"] == 0


def alone(sc, p, steps, substeps):
    out, _ = run_batch([sc], p, steps=steps, substeps=substeps)
    return out[0]


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
def test_paused_world_resumes_as_if_never_paused(solver):
    """World 1 of a batch is paused for 15 steps while the others step, then resumed: it ends
    bit for bit where the same world stepped alone for only its active steps ends, and the
    others are unaffected."""
    scs = [WORLDS[0](), WORLDS[1](), WORLDS[3]()]
    p = params(solver)
    total = sum(int(s["n"]) for s in scs)
    w = bb.World(total)
    firsts = [w.add_world(sc, *scene_bounds(sc))[1] for sc in scs]
    w.set_params(p)
    for _ in range(10):
        w.step(DT, 2)
    w.pause_world(1)
    for _ in range(15):
        w.step(DT, 2)
    w.pause_world(1, False)
    for _ in range(10):
        w.step(DT, 2)
    st = w.read_state()
    assert w.stats()["error_flags"] == 0
    w.close()
    active = {0: 35, 1: 20, 2: 35}
    for k, sc in enumerate(scs):
        ref = alone(sc, p, active[k], 2)
        n = int(sc["n"])
        for key in ref:
            assert np.array_equal(st[key][firsts[k]:firsts[k] + n], ref[key]), (k, key)


@pytest.mark.parametrize("solver", [bb.SOLVER_PGS_SOFT, bb.SOLVER_AVBD])
def test_paused_world_is_unchanged_by_a_world_added_meanwhile(solver):
    """A pile in contact with the ground is paused after 8 steps; another world joins the batch
    and the batch steps 3 times; after the pile resumes and steps twice it equals the same pile
    stepped 10 times alone (its contacts, penalties and anchors were carried untouched)."""
    a, b = scenes.pile(900, seed=4), scenes.pile(1000, seed=5)
    p = params(solver)
    w = bb.World(int(a["n"]) + int(b["n"]))
    fa = w.add_world(a, *a["bounds"])[1]
    w.set_params(p)
    for _ in range(8):
        w.step(DT, 2)
    assert w.stats()["manifold_count"] > 0
    w.pause_world(0)
    w.add_world(b, *b["bounds"])
    for _ in range(3):
        w.step(DT, 2)
    w.pause_world(0, False)
    for _ in range(2):
        w.step(DT, 2)
    st = w.read_state()
    assert w.stats()["error_flags"] == 0
    w.close()
    ref = alone(a, p, 10, 2)
    n = int(a["n"])
    for key in ref:
        assert np.array_equal(st[key][fa:fa + n], ref[key]), key


def test_refilled_slot_steps_like_a_world_added():
    """The slot of world 1 is refilled with a smaller, different scene after 10 steps: the new
    world steps bit for bit as it would alone, and the other worlds are unaffected."""
    scs = [WORLDS[0](), WORLDS[1](), WORLDS[3]()]
    new = tiny_stack()
    assert new["n"] < scs[1]["n"]
    p = params(bb.SOLVER_PGS_SOFT)
    total = sum(int(s["n"]) for s in scs)
    w = bb.World(total)
    firsts = [w.add_world(sc, *scene_bounds(sc))[1] for sc in scs]
    w.set_params(p)
    for _ in range(10):
        w.step(DT, 2)
    w.refill_world(1, new, *scene_bounds(new))
    for _ in range(12):
        w.step(DT, 2)
    st = w.read_state()
    assert w.stats()["error_flags"] == 0
    w.close()
    refs = {0: (scs[0], 22), 1: (new, 12), 2: (scs[2], 22)}
    for k, (sc, steps) in refs.items():
        ref = alone(sc, p, steps, 2)
        n = int(sc["n"])
        for key in ref:
            assert np.array_equal(st[key][firsts[k]:firsts[k] + n], ref[key]), (k, key)
    with pytest.raises(bb.BeatboxError):  # a slot holds at most its size
        w2 = bb.World(total)
        w2.add_world(new, *scene_bounds(new))
        w2.refill_world(0, scs[1], *scene_bounds(scs[1]))


@pytest.mark.parametrize("name", ["mixed_3000", "pyramids_4x300"])
def test_colour_reuse_gives_the_same_bits(name):
    """Islands whose manifolds are exactly last substep's keep last substep's colours instead of
    running the colouring rounds.  Setting the parameters before every single-substep step makes
    every colouring start afresh; both worlds must give the same bits, through piles that form
    and break apart (mixed column) and piles that settle (pyramids)."""
    sc = (scenes.mixed_column(n_bodies=3000, seed=2) if name == "mixed_3000"
          else scenes.pyramids(n_pyramids=4, boxes_per=300, gap=-0.002))
    p = params(bb.SOLVER_PGS_SOFT)
    reused = bb.world_from_scene(sc, params=p)
    fresh = bb.world_from_scene(sc, params=p)
    applied = bb.SolverParams.from_buffer_copy(bytes(fresh.params))  # with the scene's Morton box
    rounds = []
    for _ in range(160):
        reused.step(DT / 4, 1)
        fresh.set_params(applied)
        fresh.step(DT / 4, 1)
        rounds.append(reused.stats()["graph_color_rounds"])
    a, b = reused.read_state(), fresh.read_state()
    assert reused.stats()["error_flags"] == 0 and fresh.stats()["error_flags"] == 0
    assert min(rounds[40:]) < max(rounds)  # some substeps reused every island's colours
    reused.close()
    fresh.close()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
