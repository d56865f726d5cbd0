"""Scene files: a scene survives save / load unchanged (CPU); a checkpoint of a stepped world
restores its poses and velocities exactly (GPU)."""
import numpy as np
import pytest

import beatbox as bb
from beatbox import io, scenes


def test_scene_file_round_trip(tmp_path):
    for sc in (scenes.box_grid(n_side=4, layers=2), scenes.mixed_column(n_bodies=300, seed=2)):
        path = str(tmp_path / "scene.npz")
        io.save_scene(sc, path)
        back = io.load_scene(path)
        assert back["n"] == sc["n"]
        for k in ("pos", "quat", "half", "shape", "flags", "mass", "inv_inertia", "friction", "vel", "omega"):
            assert np.array_equal(back[k], sc[k]), k
        if sc.get("bounds") is not None:
            assert np.allclose(back["bounds"][0], sc["bounds"][0]) and np.allclose(back["bounds"][1], sc["bounds"][1])


@pytest.mark.gpu
def test_checkpoint_restores_the_world_state(tmp_path):
    sc = scenes.pile(300, seed=4)
    p = bb.make_params(solver=bb.SOLVER_PGS_SOFT, quirks=bb.QUIRKS_PHYSICAL)
    w = bb.world_from_scene(sc, params=p)
    for _ in range(15):
        w.step(1 / 60, 2)
    path = str(tmp_path / "ckpt.npz")
    io.save_scene(io.checkpoint(w, sc), path)
    st = w.read_state()
    w.close()
    r = bb.world_from_scene(io.load_scene(path), params=p)
    back = r.read_state()
    for k in st:
        assert np.array_equal(back[k], st[k]), k
    r.close()
