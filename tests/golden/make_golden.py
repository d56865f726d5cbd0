"""Generates tests/golden/*.npz from the oracle.

The reference repository ships no golden vectors, so these fixtures are produced by the oracle
(the CPU restatement of the reference step) and pin it against unintended changes; the CUDA
library is compared with the same oracle in the GPU tests.  Re-run after a deliberate change to
the restated algorithm:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "beat-box_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from beatbox import scenes  # noqa: E402

CASES = {
    "grid_4x3": dict(scene=lambda: scenes.box_grid(n_side=4, layers=3), solver=1, quirks=0),
    "grid_4x3_reference": dict(scene=lambda: scenes.box_grid(n_side=4, layers=3, inertia="reference", density=5.0),
                               solver=1, quirks=7),
    "mixed_400_avbd": dict(scene=lambda: scenes.mixed_column(n_bodies=400, seed=5), solver=2, quirks=0),
}
STEPS = 20


def params(case, sc):
    p = pyoracle.default_params()
    p.solver, p.quirks = case["solver"], case["quirks"]
    p.iterations = p.relax_iterations = 8
    p.avbd_iterations = 4
    if sc.get("bounds") is not None:
        p.world_min[:] = sc["bounds"][0]
        p.world_extent[:] = sc["bounds"][1]
    return p


def read(o, code, dtype):
    cnt, buf = o.debug_read(code)
    return buf[: cnt * np.dtype(dtype).itemsize].view(dtype).copy()


def generate(name):
    case = CASES[name]
    sc = case["scene"]()
    o = pyoracle.Oracle(sc, params=params(case, sc))
    o.collide(2)
    out = dict(morton=read(o, 1, np.uint32), sorted_ids=read(o, 3, np.uint32), lbvh_child=read(o, 4, np.int32),
               pairs=read(o, 7, np.uint32))
    o = pyoracle.Oracle(sc, params=params(case, sc))
    traj = []
    for _ in range(STEPS):
        o.step(1 / 60, 4)
        traj.append(o.state()["pos"])
    out["trajectory"] = np.asarray(traj)
    out["final_stats"] = np.array([o.stats()[k] for k in ("manifold_count", "contact_count", "graph_color_count")])
    return out


def main():
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **generate(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
