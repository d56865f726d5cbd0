"""Benchmark of the B200 rigid-body step (body-steps/s), one JSON line on rank 0.

Workload (default): 1,000,000 unit boxes in 1,000 pyramids of 1,000 boxes (base 18x18, tapering)
on a 32x32 grid of cells 20 m apart over a ground box, initial velocity N(0, 0.01) m/s per
component; FP32 state, dt = 1/60 s, 4 substeps, PGS_SOFT 10 solve + 10 relax iterations,
physical arithmetic (the reference's gravity / SAT-frame / inertia quirks off).  Seeded synthetic
scene (seed 0): no public dataset exists for this workload.  A "step" is one bb_step(dt, 4) of
the whole world.

Timing: the run starts from the scene at rest; W untimed warm-up steps, then the next K steps,
each bracketed by CUDA events on the world's stream (the awake settling phase of the pyramids:
every front-end, colouring and solver stage runs at full size); L2 is flushed (256 MB write)
before every timed step, outside the events.  Multi-GPU (torchrun): a single world does not
shard, so every rank steps its own replica; the time is the max over ranks and value = all
ranks' body-steps / that time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--solver pgs|avbd]
                  [--scene pyramids|mixed_column|box_grid|voxel_pile] [--mode plain|batched|served|sort]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "beat-box_b200"))

import numpy as np  # noqa: E402

from beatbox import ranks, scenes  # noqa: E402

DT = 1.0 / 60.0
SUBSTEPS = 4
L2_BYTES = 126 * 1024 * 1024
DEFAULT_BODIES = {"pyramids": 1_000_000, "mixed_column": 100_000, "box_grid": 1000, "voxel_pile": 20_000}
# DRAM bytes (read + write) of one launch, from ncu captures of the same workloads; the capture
# commands are in profiles/ (k_pgs_soft on the 100k mixed column at step ~298 of its run)
SOLVER_TRAFFIC = {("mixed_column", 100_000): 114.5e6 + 24.1e6}


def workload(args, n_bodies: int | None = None):
    """The scene and its one-line description; n_bodies overrides --bodies (samples)."""
    nb = args.bodies if n_bodies is None else n_bodies
    if args.scene == "pyramids":
        n_pyr = max(1, nb // 1000)
        sc = scenes.pyramids(n_pyramids=n_pyr, boxes_per=1000, seed=0)
        name = (f"pyramids_{n_pyr}x1000: {n_pyr} pyramids of 1000 unit boxes (base 18x18) on a 32x32 grid, "
                f"velocity N(0, 0.01) m/s, dt=1/60, {SUBSTEPS} substeps, ")
    elif args.scene == "voxel_pile":
        sc = scenes.voxel_pile(n_bodies=nb, seed=0)
        name = (f"voxel_pile_{nb // 1000}k: {nb} concave voxel bodies (L / cross / frame, "
                f"0.2 m cells, random orientation) in 3 layers over a ground box, dt=1/60, {SUBSTEPS} substeps, ")
    elif args.scene == "box_grid":
        sc = scenes.box_grid(n_side=10, seed=0)
        sc["bounds"] = ([-64.0] * 3, [128.0] * 3)  # the reference's Morton box
        name = (f"box_grid_1000: 1000 unit boxes (10x10x10, 1.1 m spacing, jitter 0.05 m, random yaw) "
                f"dropped on a ground box, dt=1/60, {SUBSTEPS} substeps, ")
    else:
        sc = scenes.mixed_column(n_bodies=nb, seed=0)
        name = (f"mixed_column_{nb // 1000}k: {nb} bodies (60% boxes / 40% spheres) in a "
                f"60x60x200 m column, 5-wall container, dt=1/60, {SUBSTEPS} substeps, ")
    if args.solver == "pgs":
        name += f"PGS_SOFT {pgs_iterations(args)} iterations ({args.schedule} schedule)"
    else:
        name += "AVBD 4 iterations (beta=10)"
    return sc, name


def run_sort(args, rank: int, local_rank: int):
    """The onesweep pair sort alone (bb_radix_sort_pairs on --sort-keys random keys): one JSON
    line with sorted keys/s and its HBM roofline (68 algorithmic bytes per key)."""
    if rank != 0:
        return
    pk = peaks()
    r = sort_roofline(local_rank, float(pk.get("hbm_gbs", 6650.0)), n=args.sort_keys, reps=max(args.steps, 1))
    print(json.dumps({"metric": "sorted keys/s", "value": r["keys"] / (r["ms_per_sort"] / 1000.0), "unit": "keys/s",
                      "n_gpus": 1, "steps": max(args.steps, 1), "warmup": 1, "higher_is_better": True,
                      "dtype": "u32", "data": "synthetic (uniform random 31-bit keys, seed 0)",
                      "config": {"workload": f"bb_radix_sort_pairs: {r['keys']} 32-bit keys + 32-bit values"},
                      "roofline": r}), flush=True)


def sort_roofline(local_rank: int, peak_gbs: float, n: int = 1 << 26, reps: int = 5) -> dict:
    """The onesweep pair sort (the step's a4 kernels, through bb_radix_sort_pairs) on 2^26 random
    32-bit keys with 32-bit values, 1 GB in and out, so every pass streams from HBM.  Algorithmic
    bytes: one histogram read of the keys (4 B/key) plus 4 passes reading and writing keys and
    values (16 B/key each), 68 B/key.  CUDA events on the stream the sort runs on; the mean of
    `reps` sorts after one warm-up sort."""
    import torch

    import beatbox as bb

    L = bb.load_library()
    dev = f"cuda:{local_rank}"
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    keys = torch.randint(0, 2 ** 31 - 1, (n,), device=dev, dtype=torch.int64, generator=g).to(torch.int32)
    vals = torch.arange(n, device=dev, dtype=torch.int32)
    ko, vo = torch.empty_like(keys), torch.empty_like(vals)
    s = torch.cuda.current_stream()
    args = [keys.data_ptr(), vals.data_ptr(), ko.data_ptr(), vo.data_ptr(), n, 32, s.cuda_stream]
    bb._check(L.bb_radix_sort_pairs(*args))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        bb._check(L.bb_radix_sort_pairs(*args))
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    ok = bool(torch.all(ko[1:].to(torch.int64) >= ko[:-1].to(torch.int64)).item())
    achieved = 68.0 * n / (ms / 1000.0) / 1e9
    return {"kernel": "k_sort_hist + 4x k_onesweep (bb_radix_sort_pairs)", "bound": "hbm", "keys": n,
            "achieved": achieved, "peak": peak_gbs, "unit": "GB/s", "frac": achieved / peak_gbs,
            "ms_per_sort": ms, "algorithmic_bytes_per_key": 68, "sorted": ok}


def run_steps(args) -> int:
    """Length of the configuration's run: 600 steps for the mixed column, 300 for the others."""
    return 600 if args.scene == "mixed_column" else 300


def pgs_iterations(args) -> int:
    """PGS solve (and relax) iterations: 8 for the 1000-box grid, 10 for the others."""
    return 8 if args.scene == "box_grid" else 10


def timed_window(args) -> int:
    """First timed step.  Pyramids: right after the W warm-up steps (the awake settling phase,
    where the sort, tree, colouring and solver work at full size).  Other scenes: centred on
    the run (their piles form as they fall), never before the W warm-up steps."""
    if args.scene == "pyramids":
        return args.warmup
    return max(args.warmup, run_steps(args) // 2 - args.steps // 2)


def solver_fields(args) -> dict:
    if args.solver == "pgs":
        return dict(solver=1, iterations=pgs_iterations(args), relax_iterations=pgs_iterations(args), quirks=0,
                    schedule=0 if args.schedule == "dataflow" else 1)
    return dict(solver=2, avbd_iterations=4, avbd_beta=10.0, quirks=0)


def sample_clocks(dev: int):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                                 "-i", str(dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except (OSError, FileNotFoundError):
        return None


def finish_clocks(proc) -> dict:
    if proc is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
        out, _ = proc.communicate()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx.append(float(f[2]))
        except ValueError:
            continue
        for k, nm in enumerate(names):
            if f[5 + k].lower().startswith("active"):
                reasons.add(nm)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def peaks() -> dict:
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        return {"hbm_gbs": 6650.0, "fallback": True}


def solver_bytes(st: dict, n: int, args) -> float:
    """Algorithmic HBM bytes of one solver launch (one substep), SoA float4 model: body
    state 64 B, props 48 B, contact row 64 B, manifold header 32 B.  PGS: the manifolds and
    contacts the colour sweeps solve (those with an awake body); AVBD: all of them."""
    if args.solver == "pgs":
        M, K = st["solved_manifolds"], st["solved_contacts"]
        it = pgs_iterations(args)
        pre = 64 * K + 4 * 32 * M + 2 * 48 * M
        sweep = 64 * K + 128 * M
        return pre + 2 * it * sweep + 128 * n
    M, K = st["manifold_count"], st["contact_count"]
    it = 4
    sweeps = it + 12 + 3  # main iterations + post-stabilisation (cascade + plain sweeps)
    return 2 * 192 * n + sweeps * (64 * n + 2 * (32 * M + 64 * K)) + it * (32 * M + 76 * K)


def cpu_sample_pyramids(args) -> int:
    return max(1, min(args.cpu_sample_pyramids, args.bodies // 1000))


def cpu_sample(args, threads: int) -> dict:
    """The step on the host cores: the oracle (a restatement of the reference's Slang passes;
    the reference itself needs Vulkan/Daxa and cannot run here) in FP32 on `threads` threads,
    over a bounded sample of the timed workload: the same steps (W untimed, then up to K timed,
    at most --cpu-budget-s seconds of them) of a world holding the first pyramids of the scene
    (their bodies start exactly as in the full world; pyramids 20 m apart never touch), or of
    the whole world for the other scenes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    pyoracle.build()
    if args.scene == "pyramids":
        n_pyr = cpu_sample_pyramids(args)
        sc, _ = workload(args, n_bodies=n_pyr * 1000)
        what = f"pyramids 0..{n_pyr - 1} of the {args.bodies // 1000} ({sc['n']} bodies with the ground)"
    else:
        sc, _ = workload(args)
        what = f"the full {sc['n']}-body world"
    p = pyoracle.default_params()
    for k, v in solver_fields(args).items():
        setattr(p, k, v)
    p.world_min[:] = sc["bounds"][0]
    p.world_extent[:] = sc["bounds"][1]
    o = pyoracle.Oracle(sc, double=False, threads=threads, params=p)
    first = timed_window(args)
    t0 = time.time()
    done = 0
    while done < first and (first - done <= args.warmup or time.time() - t0 < args.cpu_budget_s):
        o.step(DT, SUBSTEPS)
        done += 1
    t1 = time.time()
    steps = 0
    while steps < args.steps and (steps == 0 or time.time() - t1 < args.cpu_budget_s):
        o.step(DT, SUBSTEPS)
        steps += 1
    el = time.time() - t1
    v = sc["n"] * steps / el
    sample = (f"steps {done}..{done + steps - 1} (the timed window starts at step {first}) of {what}, "
              f"FP32 oracle, {threads} threads")
    return {"value": v, "unit": "body-steps/s", "cores": threads, "kind": "port", "sample": sample,
            "steps": steps, "first_step": done, "same_steps": done == first and steps == args.steps,
            "ms_per_step": 1000 * el / max(steps, 1), "bodies": int(sc["n"])}


def run_reference(args, rank: int, world_size: int):
    """Times the reference's CPU implementation of the step on the host cores (all threads):
    the oracle port, on a bounded sample of this bench's workload and step window."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    _, name = workload(args)
    cb = cpu_sample(args, threads)
    v = cb["value"]
    line = {"impl": "reference", "metric": "body-steps/s", "value": v, "unit": "body-steps/s", "n_gpus": world_size,
            "steps": cb["steps"], "warmup": cb["first_step"], "ms_per_step": cb["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene, seed 0)",
            "config": {"workload": name, "bodies": int(workload(args)[0]["n"]), "substeps": SUBSTEPS, "dt": DT,
                       "timed_steps": f"steps {timed_window(args)}..{timed_window(args) + args.steps - 1}"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "same_steps")},
            "e2e": {"value": v, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def make_world(bb, args, sc, local_rank: int):
    # a voxel pair takes six manifold slots (one per face direction)
    w = bb.World(sc["n"], pairs_per_body=64 if args.scene == "voxel_pile" else 16, device=local_rank)
    w.add_scene(sc)
    p = bb.default_params()
    p.world_min[:] = sc["bounds"][0]
    p.world_extent[:] = sc["bounds"][1]
    w.set_params(p, **solver_fields(args))
    return w


def time_steps(torch, w, steps: int, flush, dev: str):
    """Device time (ms) of each of `steps` steps: CUDA events on the world's stream, L2 flushed
    (outside the events) before each."""
    stream = torch.cuda.ExternalStream(w.stream, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        evs[k][0].record(stream)
        w.step(DT, SUBSTEPS)
        evs[k][1].record(stream)
    w.sync()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def kernel_roof(kernel: str, bytes_total: float, ms_total: float, launches: int, peak_gbs: float, traffic=None,
                model: str = "") -> dict:
    achieved = bytes_total / (ms_total / 1000.0) / 1e9 if ms_total > 0 else 0.0
    return {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
            "frac": achieved / peak_gbs, "traffic": traffic,
            "algorithmic_bytes_per_launch": bytes_total / max(launches, 1),
            "ms_per_launch": ms_total / max(launches, 1), "launches": launches, "model": model}


def profiled_window(bb, args, sc, local_rank: int, first: int, steps: int, peak_gbs: float, traffic=None) -> dict:
    """A second world with the same deterministic history, profiled over the timed steps:
    per-stage CUDA-event times (a substep run stage by stage with events between) and the
    rooflines of the solver, the sort and the refit from their own event times and the
    algorithmic bytes of the same substeps (live counts after each step)."""
    w = make_world(bb, args, sc, local_rank)
    for _ in range(first):
        w.step(DT, SUBSTEPS)
    w.sync()
    n = w.n
    n_dyn = int(w.stats()["active_body_count"])
    w.set_profiling(True)
    solve_b = sort_b = refit_b = 0.0
    front_runs = 0
    for _ in range(steps):
        w.step(DT, SUBSTEPS)
        st = w.stats()
        solve_b += SUBSTEPS * solver_bytes(st, n, args)
        if st["sleeping_count"] < n_dyn:  # the front end ran (it is skipped once every body sleeps)
            front_runs += SUBSTEPS
    stages = w.stage_times()
    w.set_profiling(False)
    w.close()
    sort_b, refit_b = 68.0 * n * front_runs, 52.0 * n * front_runs
    subs = steps * SUBSTEPS
    solver_name = "k_pgs_soft" if args.solver == "pgs" else "AVBD kernels"
    roofs = {
        "solve": kernel_roof(f"solve ({solver_name})", solve_b, stages.get("solve", 0.0), subs, peak_gbs, traffic,
                             "PGS_SOFT: pre-step 64K + 224M, each of 2I sweeps 64K + 128M, integrate 128N bytes "
                             "(K contacts, M manifolds solved this substep)"),
        "sort": kernel_roof("sort (k_sort_hist + 4x k_onesweep)", sort_b, stages.get("sort", 0.0), max(front_runs, 1),
                            peak_gbs, None, "68 B per body: histogram read 4 B + 4 passes x 16 B"),
        "refit": kernel_roof("refit (k_refit, node records fused)", refit_b, stages.get("refit", 0.0),
                             max(front_runs, 1), peak_gbs, None, "52 B per body: leaf boxes read 24 B, internal "
                             "boxes written 24 B, parents 4 B"),
    }
    return {"stage_ms_per_substep": {k: v / subs for k, v in stages.items()}, "rooflines": roofs,
            "front_end_substeps": front_runs}


def run_ours(args, rank: int, world_size: int, local_rank: int):
    import torch

    import beatbox as bb

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    sc, name = workload(args)
    first = timed_window(args)
    pk = peaks()
    peak_gbs = float(pk.get("hbm_gbs", 6650.0))
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    w = make_world(bb, args, sc, local_rank)
    for _ in range(first):  # the W warm-up steps (and, for the other scenes, the pre-roll)
        w.step(DT, SUBSTEPS)
    w.sync()
    n = w.n
    launches0 = w.launches()
    clocks = sample_clocks(local_rank)
    if dist is not None:
        dist.barrier()
    ms = time_steps(torch, w, args.steps, flush, dev)
    clk = finish_clocks(clocks)
    total_ms = sum(ms)
    launches = w.launches() - launches0
    stats = w.stats()
    t = torch.tensor([total_ms], device=dev)
    if dist is not None:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world_size * n * args.steps / (max_ms / 1000.0)

    extras = {}
    if world_size == 1 and args.scene == "pyramids" and not args.no_extras:
        # the same world later in its run, once every body sleeps (front end skipped, frozen
        # pairs carried, no island coloured): steps 145..154 of the 300-step run
        done = first + args.steps
        for _ in range(max(0, 145 - done)):
            w.step(DT, SUBSTEPS)
        w.sync()
        sms = time_steps(torch, w, 10, flush, dev)
        extras["asleep_window"] = {"value": n * 10 / (sum(sms) / 1000.0), "unit": "body-steps/s",
                                   "ms_per_step": sum(sms) / 10, "steps": f"steps {max(done, 145)}..{max(done, 145) + 9}",
                                   "sleeping_count": w.stats()["sleeping_count"]}
    w.close()

    # end to end through the public API with pinned host buffers: upload state, step, read back,
    # over the same steps (a second world with the same deterministic history)
    w2 = make_world(bb, args, sc, local_rank)
    for _ in range(first):
        w2.step(DT, SUBSTEPS)
    w2.sync()
    pin = lambda shape: torch.empty(shape, dtype=torch.float32).pin_memory().numpy()  # noqa: E731
    st0 = w2.read_state()
    host = {k: pin(v.shape) for k, v in st0.items()}
    for k in host:
        host[k][...] = st0[k]
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        w2.write_state(host["pos"], host["quat"], host["vel"], host["omega"])
        w2.step(DT, SUBSTEPS)
        w2.read_state(host)
    e2e_s = time.perf_counter() - t0
    w2.close()
    e2e_t = torch.tensor([e2e_s], device=dev)
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world_size * n * args.steps / float(e2e_t.item())
    io_bytes = n * (12 + 16 + 12 + 12)

    # per-stage split and per-kernel rooflines on the timed steps
    prof = profiled_window(bb, args, sc, local_rank, first, args.steps, peak_gbs,
                           SOLVER_TRAFFIC.get((args.scene, args.bodies)) if args.solver == "pgs" else None)
    stage = prof["stage_ms_per_substep"]
    dom = max(stage, key=stage.get) if stage else "solve"
    roof = dict(prof["rooflines"]["solve"])
    roof.update({"peak_source": "measured" if not pk.get("fallback") else "fallback",
                 "stage_ms_per_substep": stage, "dominant_stage": dom})

    if world_size == 1 and args.scene == "pyramids" and not args.no_extras:
        # config 2 beside it: the 100k mixed column at the centre of its 600-step run
        class A:  # noqa: N801
            pass

        a2 = A()
        a2.__dict__.update(vars(args))
        a2.scene, a2.bodies = "mixed_column", DEFAULT_BODIES["mixed_column"]
        sc2, name2 = workload(a2)
        f2 = timed_window(a2)
        wc = make_world(bb, a2, sc2, local_rank)
        for _ in range(f2):
            wc.step(DT, SUBSTEPS)
        wc.sync()
        ms2 = time_steps(torch, wc, args.steps, flush, dev)
        wc.close()
        p2 = profiled_window(bb, a2, sc2, local_rank, f2, args.steps, peak_gbs,
                             SOLVER_TRAFFIC.get((a2.scene, a2.bodies)))
        extras["mixed_column_100k"] = {"workload": name2, "value": sc2["n"] * args.steps / (sum(ms2) / 1000.0),
                                       "unit": "body-steps/s", "ms_per_step": sum(ms2) / args.steps,
                                       "timed_steps": f"steps {f2}..{f2 + args.steps - 1} of the 600-step run",
                                       "stage_ms_per_substep": p2["stage_ms_per_substep"],
                                       "rooflines": p2["rooflines"]}

    sort_roof = sort_roofline(local_rank, peak_gbs) if rank == 0 and not args.no_extras else None

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(args, os.cpu_count() or 1)
    if rank == 0:
        line = {"metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world_size,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded scene, seed 0)",
                "config": {"workload": name, "bodies": n, "substeps": SUBSTEPS, "dt": DT,
                           "parallelism": f"replicas x{world_size}", "l2": "flushed before every timed step",
                           "timed_steps": f"steps {first}..{first + args.steps - 1} of the {run_steps(args)}-step run "
                                          f"(after {first} untimed steps from rest, the last {args.warmup} of them "
                                          f"the warm-up)"},
                "e2e": {"value": e2e_value, "unit": "body-steps/s", "h2d_bytes_per_step": io_bytes,
                        "d2h_bytes_per_step": io_bytes, "steps": args.steps,
                        "what": "bb_write_state + bb_step + bb_read_state with pinned host buffers, same steps"},
                "gpu_launches": launches, "roofline": roof, "rooflines": prof["rooflines"],
                "sort_roofline": sort_roof, "cpu_baseline": cpu, "clocks": clk,
                "ms_per_timed_step": [round(x, 3) for x in ms], "step_stats": stats, **extras}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def batched_scenes(n_worlds: int):
    """Config-4 batch: world k is a pile of floor(exp(U(ln 16, ln 2048))) bodies, seed k + 1."""
    sizes = scenes.batch_sizes(n_worlds, seed=0)
    return [scenes.pile(int(nw), seed=k + 1) for k, nw in enumerate(sizes)]


def run_batched(args, rank: int, world_size: int, local_rank: int):
    """Config 4: thousands of independent worlds stepped as one batch (world-prefixed Morton
    keys, one CUDA-graph launch per step), against the same worlds stepped one at a time through
    the plain single-world path with the same kernels."""
    import torch

    import beatbox as bb

    torch.cuda.set_device(local_rank)
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    all_scs = batched_scenes(args.worlds)
    sizes = [int(sc["n"]) for sc in all_scs]
    scs = [all_scs[k] for k in ranks.balanced_share(sizes, rank, world_size)]
    total = sum(int(sc["n"]) for sc in scs)
    p = bb.make_params(solver=bb.SOLVER_PGS_SOFT, iterations=8, relax_iterations=8, quirks=bb.QUIRKS_PHYSICAL)
    w = bb.World(total, pairs_per_body=8, device=local_rank)
    for sc in scs:
        w.add_world(sc, *sc["bounds"])
    w.set_params(p)
    run = 120
    first = max(args.warmup, run // 2 - args.steps // 2)
    tune = w.autotune(DT, SUBSTEPS, trial_steps=1)  # its trial steps are ordinary steps of the run
    tuned = w.stats()["substeps_run"] // SUBSTEPS
    for _ in range(max(0, first - tuned)):
        w.step(DT, SUBSTEPS)
    w.sync()
    done = max(first, tuned)
    stream = torch.cuda.ExternalStream(w.stream)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
    clocks = sample_clocks(local_rank)
    launches0 = w.launches()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        evs[k][0].record(stream)
        w.step(DT, SUBSTEPS)
        evs[k][1].record(stream)
    w.sync()
    torch.cuda.synchronize()
    clk = finish_clocks(clocks)
    batch_ms = sum(a.elapsed_time(b) for a, b in evs)
    launches = w.launches() - launches0
    st = w.stats()
    t = torch.tensor([batch_ms], device=f"cuda:{local_rank}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = sum(sizes) * args.steps / (float(t.item()) / 1000.0)

    # end to end: upload all worlds' state, step, read it back (pinned host buffers)
    host = {k: torch.empty(v.shape, dtype=torch.float32).pin_memory().numpy() for k, v in w.read_state().items()}
    for k, v in w.read_state().items():
        host[k][...] = v
    t0 = time.perf_counter()
    e2e_steps = min(args.steps, 20)
    for _ in range(e2e_steps):
        w.write_state(host["pos"], host["quat"], host["vel"], host["omega"])
        w.step(DT, SUBSTEPS)
        w.read_state(host)
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], device=f"cuda:{local_rank}")
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = sum(sizes) * e2e_steps / float(e2e_t.item())
    # per-stage CUDA-event split over a few profiled steps (after the timed and end-to-end runs)
    prof_steps = max(1, min(args.steps, 5))
    w.set_profiling(True)
    for _ in range(prof_steps):
        w.step(DT, SUBSTEPS)
    w.sync()
    stages = {k: v / (prof_steps * SUBSTEPS) for k, v in w.stage_times().items()}
    w.set_profiling(False)
    w.close()

    # plain path: every plain_stride-th of this rank's worlds alone, same kernels, same step window
    plain_bodies = 0
    plain_ms = 0.0
    ks = 3
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for sc in scs[:: args.plain_stride]:
        pw = bb.world_from_scene(sc, params=p, pairs_per_body=8)
        for _ in range(done):
            pw.step(DT, SUBSTEPS)
        pw.sync()
        ps = torch.cuda.ExternalStream(pw.stream)
        ev0.record(ps)
        for _ in range(ks):
            pw.step(DT, SUBSTEPS)
        ev1.record(ps)
        pw.sync()
        plain_ms += ev0.elapsed_time(ev1)
        plain_bodies += int(sc["n"]) * ks
        pw.close()
    plain_value = plain_bodies / (plain_ms / 1000.0) if plain_ms > 0 else None
    if rank == 0:
        line = {"metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world_size,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(t.item()) / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded piles, seeds 1..worlds)",
                "config": {"workload": f"batched_{args.worlds}: {args.worlds} worlds of floor(exp(U(ln 16, ln 2048))) "
                                       f"bodies ({sum(sizes)} in total), config-1 piles (60% unit boxes / 40% "
                                       f"spheres r=0.5) each over its own ground, dt=1/60, {SUBSTEPS} substeps, "
                                       "PGS_SOFT 8 iterations, autotuned",
                           "worlds": args.worlds, "bodies": sum(sizes), "parallelism": f"worlds split over {world_size} GPU(s)",
                           "l2": "flushed before every timed step",
                           "timed_steps": f"steps {done}..{done + args.steps - 1} of the {run}-step run",
                           "tuning": tune},
                "plain": {"value": plain_value, "unit": "body-steps/s",
                          "sample": f"every {args.plain_stride}th world alone through the single-world path, "
                                    f"{ks} steps each after the same {done}-step roll, device time"},
                "batched_over_plain": (value / world_size) / plain_value if plain_value else None,
                "e2e": {"value": e2e_value, "unit": "body-steps/s", "h2d_bytes_per_step": total * 52,
                        "d2h_bytes_per_step": total * 52, "steps": e2e_steps,
                        "what": "bb_write_state + bb_step + bb_read_state of the whole batch, pinned host buffers"},
                "gpu_launches": launches, "clocks": clk, "step_stats": st,
                "stage_ms_per_substep": stages}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_served(args, rank: int, world_size: int, local_rank: int):
    """Config 5: Poisson arrivals of step requests for worlds of 64..50,000 bodies (log-uniform;
    config-1 piles), 1..120 steps each, PGS_SOFT or AVBD 50/50, half of them creating a world and
    half continuing an existing one; worlds stay on the device between requests, admission by a
    120 GB HBM budget.  For each arrival rate a fixed number of requests is submitted in real time
    and served to completion; throughput and p50/p99 request latency are reported per rate.  The
    server batches continuously: worlds of one size and step class are slots of one batched
    world, and every step of a batch advances all of its running requests."""
    import numpy as np
    import torch

    import beatbox as bb

    torch.cuda.set_device(local_rank)
    rng = np.random.default_rng(5)
    n_templates = 48
    sizes = np.floor(np.exp(rng.uniform(np.log(64), np.log(50000), n_templates))).astype(int)
    templates = [scenes.pile(int(nb), seed=200 + k) for k, nb in enumerate(sizes)]
    arrays = [bb.scene_request_arrays(sc) for sc in templates]
    p_pgs = bb.make_params(solver=bb.SOLVER_PGS_SOFT, iterations=10, relax_iterations=10, quirks=bb.QUIRKS_PHYSICAL)
    p_avbd = bb.make_params(solver=bb.SOLVER_AVBD, avbd_iterations=4, avbd_beta=10.0, quirks=bb.QUIRKS_PHYSICAL)
    srv = bb.Server(hbm_budget_bytes=120 << 30, max_active=args.max_active, pairs_per_body=16, device=local_rank)
    clocks = sample_clocks(local_rank)
    rates = [float(x) for x in args.rates.split(",")]
    per_rate = []
    next_key = 1
    known = []  # (key, template) of worlds created so far
    for lam in rates:
        tickets = []
        bodies = 0
        submit_s = []
        t_start = time.perf_counter()
        t_next = t_start
        for _ in range(args.requests):
            t_next += rng.exponential(1.0 / lam)
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            steps = int(rng.integers(1, 121))
            params = p_pgs if rng.random() < 0.5 else p_avbd
            if not known or rng.random() < 0.5:
                k = int(rng.integers(0, n_templates))
                key = next_key
                next_key += 1
                known.append((key, k))
                t_call = time.perf_counter()
                tk = srv.submit(key, steps, params, DT, SUBSTEPS, scene=templates[k], arrays=arrays[k])
            else:
                key, k = known[int(rng.integers(0, len(known)))]
                t_call = time.perf_counter()
                tk = srv.submit(key, steps, params, DT, SUBSTEPS)
            submit_s.append(time.perf_counter() - t_call)
            tickets.append(tk)
            bodies += int(templates[k]["n"]) * steps
        res = [srv.wait(t) for t in tickets]
        ok = [r for r in res if r["result"] == bb.OK]
        lat = np.array([r["finish_s"] - r["submit_s"] for r in ok])
        span = max(r["finish_s"] for r in res) - min(r["submit_s"] for r in res)
        codes: dict = {}
        flags: dict = {}
        for r in res:
            if r["result"] != bb.OK:
                codes[str(r["result"])] = codes.get(str(r["result"]), 0) + 1
                fk = f'{r["error_flags"]}@{r["error_site"]}'
                flags[fk] = flags.get(fk, 0) + 1
        per_rate.append({"rate_req_s": lam, "requests": len(res), "failed": len(res) - len(ok), "fail_codes": codes,
                         "fail_error_flags_at_site": flags,
                         "body_steps_per_s": bodies / span if span > 0 else None,
                         "p50_ms": float(np.percentile(lat, 50) * 1000) if len(lat) else None,
                         "p99_ms": float(np.percentile(lat, 99) * 1000) if len(lat) else None,
                         "submit_window_s": time.perf_counter() - t_start,
                         "submit_call_ms_max": 1000 * max(submit_s),
                         "queue_wait_ms_p50": float(np.percentile([r["start_s"] - r["submit_s"] for r in res], 50) * 1000),
                         "run_ms_p50": float(np.percentile([r["finish_s"] - r["start_s"] for r in res], 50) * 1000)})
        print(json.dumps({"progress": per_rate[-1], "server": srv.stats()}), file=sys.stderr, flush=True)
    clk = finish_clocks(clocks)
    st = srv.stats()
    srv.close()
    best = max(per_rate, key=lambda r: r["body_steps_per_s"] or 0)
    line = {"metric": "body-steps/s", "value": best["body_steps_per_s"], "unit": "body-steps/s", "n_gpus": 1,
            "steps": args.requests, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded piles and arrivals)",
            "config": {"workload": "served: Poisson arrivals, worlds of floor(exp(U(ln 64, ln 50000))) bodies "
                                   "(config-1 piles), 1..120 steps per request, PGS_SOFT 10 / AVBD 4 50/50, half new "
                                   "worlds, 120 GB HBM budget, dt=1/60, 4 substeps",
                       "rates_req_s": rates, "requests_per_rate": args.requests, "max_active": args.max_active},
            "per_rate": per_rate, "server": st, "clocks": clk,
            "value_is": "the best per-rate throughput (body-steps of the requests / first submit to last finish)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solver", default="pgs", choices=["pgs", "avbd"])
    ap.add_argument("--bodies", type=int, default=None, help="bodies of the scene (default: its configuration's)")
    ap.add_argument("--scene", default="pyramids", choices=["pyramids", "mixed_column", "box_grid", "voxel_pile"],
                    help="pyramids: bodies/1000 box pyramids (default, 1M boxes); mixed_column: the 100k mixed "
                         "column; box_grid: the 1000-box grid; voxel_pile: concave voxel bodies")
    ap.add_argument("--schedule", default="barrier", choices=["dataflow", "barrier"],
                    help="PGS schedule: per-body dataflow counters or a grid barrier per colour")
    ap.add_argument("--mode", default="plain", choices=["plain", "batched", "served", "sort"],
                    help="plain: one world (default); batched: config-4 batch of independent worlds; "
                         "served: config-5 serving loop; sort: the a4 pair sort alone on --sort-keys keys")
    ap.add_argument("--sort-keys", type=int, default=1 << 26)
    ap.add_argument("--rates", default="200,500,1000,2000,5000")
    ap.add_argument("--requests", type=int, default=200, help="requests per arrival rate (served mode)")
    ap.add_argument("--max-active", type=int, default=1024, help="requests in flight at once (served mode)")
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--plain-stride", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the asleep window, config 2 and the sort alone")
    ap.add_argument("--cpu-sample-pyramids", type=int, default=16,
                    help="pyramids in the CPU baseline's sample world (pyramids scene)")
    ap.add_argument("--cpu-budget-s", type=float, default=60.0, help="bound on the CPU baseline's timed steps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.bodies is None:
        args.bodies = DEFAULT_BODIES[args.scene]
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world_size)
    elif args.mode == "batched":
        run_batched(args, rank, world_size, local_rank)
    elif args.mode == "served":
        if rank == 0:
            run_served(args, rank, world_size, local_rank)
    elif args.mode == "sort":
        run_sort(args, rank, local_rank)
    else:
        run_ours(args, rank, world_size, local_rank)


if __name__ == "__main__":
    main()
