"""Benchmark of the B200 rigid-body step (body-steps/s), one JSON line on rank 0.

Workload (default): 100,000 mixed bodies (60% boxes with half extents U[0.2, 0.8], 40% spheres
with lognormal radii) dropped from a 60x60x200 m column into a 5-wall container; FP32 state,
dt = 1/60 s, 4 substeps, PGS_SOFT 10 solve + 10 relax iterations, physical arithmetic (the
reference's gravity / SAT-frame / inertia quirks off).  Synthetic seeded scene (seed 0): no
public dataset exists for this workload.  A "step" is one bb_step(dt, 4) of the whole world.

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events on the world's
stream; L2 is flushed (256 MB write) before every timed step, outside the events.  Multi-GPU
(torchrun): a single world does not shard, so every rank steps its own replica; the time is
the max over ranks and value = all ranks' body-steps / that time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--solver pgs|avbd]
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
N_BODIES = 100_000
L2_BYTES = 126 * 1024 * 1024
# DRAM bytes (read + write) of one k_pgs_soft launch on the 100k mixed column, from one ncu
# capture at step ~298 of the run (dram__bytes_read.sum + dram__bytes_write.sum; the capture
# command is in profiles/k_pgs_soft_k_narrow_k_components_mixed_column_100k.md)
SOLVER_TRAFFIC_MIXED_100K = 114.5e6 + 24.1e6


def workload(args):
    if args.scene == "pyramids":
        n_pyr = max(1, args.bodies // 1000)
        sc = scenes.pyramids(n_pyramids=n_pyr, boxes_per=1000, seed=0)
        name = (f"pyramids_{n_pyr}x1000: {n_pyr} pyramids of 1000 unit boxes (base 18x18) on a 32x32 grid, "
                f"velocity N(0, 0.01) m/s, dt=1/60, {SUBSTEPS} substeps, ")
    elif args.scene == "voxel_pile":
        sc = scenes.voxel_pile(n_bodies=args.bodies, seed=0)
        name = (f"voxel_pile_{args.bodies // 1000}k: {args.bodies} concave voxel bodies (L / cross / frame, "
                f"0.2 m cells, random orientation) in 3 layers over a ground box, dt=1/60, {SUBSTEPS} substeps, ")
    elif args.scene == "box_grid":
        sc = scenes.box_grid(n_side=10, seed=0)
        sc["bounds"] = ([-64.0] * 3, [128.0] * 3)  # the reference's Morton box
        name = (f"box_grid_1000: 1000 unit boxes (10x10x10, 1.1 m spacing, jitter 0.05 m, random yaw) "
                f"dropped on a ground box, dt=1/60, {SUBSTEPS} substeps, ")
    else:
        sc = scenes.mixed_column(n_bodies=args.bodies, seed=0)
        name = (f"mixed_column_{args.bodies // 1000}k: {args.bodies} bodies (60% boxes / 40% spheres) in a "
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
    """First timed step: centred on the run, never before the W warm-up steps."""
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
    state 64 B, props 48 B, contact row 64 B, manifold header 32 B."""
    M, K = st["manifold_count"], st["contact_count"]
    if args.solver == "pgs":
        it = 10
        pre = 64 * K + 4 * 32 * M + 2 * 48 * M
        sweep = 64 * K + 128 * M
        return pre + 2 * it * sweep + 128 * n
    it = 4
    sweeps = it + 12 + 3  # main iterations + post-stabilisation (cascade + plain sweeps)
    return 2 * 192 * n + sweeps * (64 * n + 2 * (32 * M + 64 * K)) + it * (32 * M + 76 * K)


def run_reference(args, rank: int, world_size: int):
    """Times the reference's CPU implementation of the step: the oracle (a restatement of the
    reference's Slang passes; the reference itself needs Vulkan/Daxa and cannot run here) in
    FP32 on all host cores."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    pyoracle.build()
    sc, name = workload(args)
    threads = os.cpu_count() or 1
    p = pyoracle.default_params()
    for k, v in solver_fields(args).items():
        setattr(p, k, v)
    p.world_min[:] = sc["bounds"][0]
    p.world_extent[:] = sc["bounds"][1]
    o = pyoracle.Oracle(sc, double=False, threads=threads, params=p)
    budget = args.ref_budget_s
    first = timed_window(args)
    t0 = time.time()
    done = 0  # untimed steps: pre-roll to the timed window (bounded by the budget), then warm-up
    while done < first and (first - done <= args.warmup or time.time() - t0 < budget):
        o.step(DT, SUBSTEPS)
        done += 1
    t1 = time.time()
    steps = 0
    while steps < args.steps:
        o.step(DT, SUBSTEPS)
        steps += 1
        if time.time() - t1 > budget:
            break
    el = time.time() - t1
    v = sc["n"] * steps / el
    sample = (f"steps {done}..{done + steps - 1} of the {run_steps(args)}-step run ({steps} of the {args.steps} "
              f"timed steps; the window starts at step {first}, fewer if the {budget:.0f} s pre-roll budget ran out) "
              f"of the full {sc['n']}-body world, FP32 oracle, {threads} threads")
    warm = done
    line = {"impl": "reference", "metric": "body-steps/s", "value": v, "unit": "body-steps/s", "n_gpus": world_size,
            "steps": steps, "warmup": warm, "ms_per_step": 1000 * el / max(steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "config": {"workload": name, "bodies": sc["n"], "substeps": SUBSTEPS, "dt": DT},
            "cpu_baseline": {"value": v, "unit": "body-steps/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world_size: int, local_rank: int):
    import torch

    import beatbox as bb

    torch.cuda.set_device(local_rank)
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    sc, name = workload(args)
    fields = solver_fields(args)

    def make_world():
        # a voxel pair takes six manifold slots (one per face direction)
        w = bb.World(sc["n"], pairs_per_body=64 if args.scene == "voxel_pile" else 16, device=local_rank)
        w.add_scene(sc)
        p = bb.default_params()
        p.world_min[:] = sc["bounds"][0]
        p.world_extent[:] = sc["bounds"][1]
        w.set_params(p, **fields)
        return w

    # The configuration is a run of RUN_STEPS steps whose cost per step grows as the pile forms;
    # K timed steps are centred on that run (untimed pre-roll first), so a short K still
    # measures a representative part of it, and K >= RUN_STEPS - W times the whole run.
    first = timed_window(args)

    def roll(world):
        for _ in range(first):
            world.step(DT, SUBSTEPS)
        world.sync()

    w = make_world()
    stream = torch.cuda.ExternalStream(w.stream)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
    roll(w)
    warm_state = w.read_state()
    warm_flags = w.read_flags()
    n = w.n
    launches0 = w.launches()
    clocks = sample_clocks(local_rank)
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
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    launches = w.launches() - launches0
    stats = w.stats()
    t = torch.tensor([total_ms], device=f"cuda:{local_rank}")
    if dist is not None:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world_size * n * args.steps / (max_ms / 1000.0)

    # end to end through the public API with pinned host buffers: upload state, step, read back
    w2 = make_world()
    roll(w2)  # the same deterministic history: both measurements cover the same steps
    pin = lambda shape: torch.empty(shape, dtype=torch.float32).pin_memory().numpy()  # noqa: E731
    host = {k: pin(v.shape) for k, v in warm_state.items()}
    for k in host:
        host[k][...] = w2.read_state()[k]
    e2e_steps = args.steps  # the same steps as the device-timed run
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        w2.write_state(host["pos"], host["quat"], host["vel"], host["omega"])
        w2.step(DT, SUBSTEPS)
        w2.read_state(host)
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], device=f"cuda:{local_rank}")
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world_size * n * e2e_steps / float(e2e_t.item())
    io_bytes = n * (12 + 16 + 12 + 12)
    w2.close()

    # roofline of the dominant stage: per-stage CUDA-event times over a profiled pass
    prof_steps = max(1, min(args.steps, 20))
    w.set_profiling(True)
    for _ in range(prof_steps):
        w.step(DT, SUBSTEPS)
    w.sync()
    stages = w.stage_times()
    w.set_profiling(False)
    st_now = w.stats()
    launches_per_stage = prof_steps * SUBSTEPS
    dom = max(stages, key=stages.get) if stages else "solve"
    pk = peaks()
    peak_gbs = float(pk.get("hbm_gbs", 6650.0))
    solve_ms = stages.get("solve", 0.0) / launches_per_stage
    sb = solver_bytes(st_now, n, args)
    achieved = sb / (solve_ms / 1000.0) / 1e9 if solve_ms > 0 else 0.0
    roof = {"kernel": "solve (k_pgs_soft)" if args.solver == "pgs" else "solve (AVBD kernels)", "bound": "hbm",
            "achieved": achieved, "peak": peak_gbs, "unit": "GB/s", "frac": achieved / peak_gbs,
            "peak_source": "measured" if not pk.get("fallback") else "fallback",
            "traffic": (SOLVER_TRAFFIC_MIXED_100K if args.solver == "pgs" and args.scene == "mixed_column"
                        and args.bodies == N_BODIES else None),
            "algorithmic_bytes_per_launch": sb, "ms_per_launch": solve_ms,
            "stage_ms_per_substep": {k: v / launches_per_stage for k, v in stages.items()}, "dominant_stage": dom}

    sort_roof = sort_roofline(local_rank, peak_gbs) if rank == 0 else None

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, sc, warm_state, warm_flags)
    if rank == 0:
        line = {"metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world_size,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded scene, seed 0)",
                "config": {"workload": name, "bodies": n, "substeps": SUBSTEPS, "dt": DT,
                           "parallelism": f"replicas x{world_size}", "l2": "flushed before every timed step",
                           "timed_steps": f"steps {first}..{first + args.steps - 1} of the {run_steps(args)}-step run "
                                          f"(the last {args.warmup} untimed steps before them are the warm-up)"},
                "e2e": {"value": e2e_value, "unit": "body-steps/s", "h2d_bytes_per_step": io_bytes,
                        "d2h_bytes_per_step": io_bytes, "steps": e2e_steps,
                        "what": "bb_write_state + bb_step + bb_read_state with pinned host buffers"},
                "gpu_launches": launches, "roofline": roof, "sort_roofline": sort_roof, "cpu_baseline": cpu,
                "clocks": clk,
                "step_stats": stats}
        print(json.dumps(line), flush=True)
    w.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(args, sc, state, flags) -> dict:
    """Oracle (FP32, all host threads) continued from the GPU's post-warm-up state for about
    15 s of CPU time: a bounded sample of the timed workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    pyoracle.build()
    sc2 = dict(sc)
    sc2["pos"], sc2["quat"], sc2["vel"], sc2["omega"] = state["pos"], state["quat"], state["vel"], state["omega"]
    sc2["flags"] = flags
    threads = os.cpu_count() or 1
    p = pyoracle.default_params()
    for k, v in solver_fields(args).items():
        setattr(p, k, v)
    p.world_min[:] = sc["bounds"][0]
    p.world_extent[:] = sc["bounds"][1]
    o = pyoracle.Oracle(sc2, double=False, threads=threads, params=p)
    t0 = time.time()
    steps = 0
    while steps < args.steps and (steps == 0 or time.time() - t0 < 15.0):
        o.step(DT, SUBSTEPS)
        steps += 1
    el = time.time() - t0
    return {"value": sc["n"] * steps / el, "unit": "body-steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} steps of the {sc['n']}-body world continued from the GPU state after "
                      f"{args.warmup} warm-up steps (cold warm start), FP32 oracle"}


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
    and served to completion; throughput and p50/p99 request latency are reported per rate."""
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
        for r in res:
            if r["result"] != bb.OK:
                codes[str(r["result"])] = codes.get(str(r["result"]), 0) + 1
        per_rate.append({"rate_req_s": lam, "requests": len(res), "failed": len(res) - len(ok), "fail_codes": codes,
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
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solver", default="pgs", choices=["pgs", "avbd"])
    ap.add_argument("--bodies", type=int, default=N_BODIES)
    ap.add_argument("--scene", default="mixed_column", choices=["mixed_column", "pyramids", "box_grid", "voxel_pile"],
                    help="mixed_column: the 100k mixed column (default); pyramids: bodies/1000 box pyramids; "
                         "box_grid: the 1000-box grid; voxel_pile: concave voxel bodies")
    ap.add_argument("--schedule", default="barrier", choices=["dataflow", "barrier"],
                    help="PGS schedule: per-body dataflow counters or a grid barrier per colour")
    ap.add_argument("--mode", default="plain", choices=["plain", "batched", "served", "sort"],
                    help="plain: one world (default); batched: config-4 batch of independent worlds; "
                         "served: config-5 serving loop; sort: the a4 pair sort alone on --sort-keys keys")
    ap.add_argument("--sort-keys", type=int, default=1 << 26)
    ap.add_argument("--rates", default="200,500,1000,2000,5000")
    ap.add_argument("--requests", type=int, default=60, help="requests per arrival rate (served mode)")
    ap.add_argument("--max-active", type=int, default=8)
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--plain-stride", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=150.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
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
