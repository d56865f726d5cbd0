"""The reference's demo scenes 1..7 (src/scene_manager.hpp:114-823) as shipped data files: each
file equals its builder in beatbox.reference_scenes array for array, and the scenes have the
reference's bodies (counts, static bodies, masses, the box pool's hashed layout)."""
import math

import numpy as np
import pytest

from beatbox import io, reference_scenes, scenes


@pytest.mark.parametrize("k", range(1, 8))
def test_data_file_equals_builder(k):
    a, b = io.load_reference_scene(k), reference_scenes.reference_scene(k)
    assert a["n"] == b["n"]
    for key in io._ARRAYS + io._OPTIONAL:
        assert np.array_equal(a[key], b[key]), key
    assert len(a.get("voxel_shapes", [])) == len(b.get("voxel_shapes", []))
    for va, vb in zip(a.get("voxel_shapes", []), b.get("voxel_shapes", [])):
        assert np.array_equal(va["solid"], vb["solid"]) and va["voxel_size"] == vb["voxel_size"]


def test_scene_counts_and_statics():
    want = {1: (19, 1), 2: (1001, 1), 3: (27, 2), 4: (17, 4), 5: (12, 3), 6: (12, 3), 7: (438, 6)}
    for k, (n, statics) in want.items():
        sc = io.load_reference_scene(k)
        dyn = (sc["flags"] & scenes.BODY_DYNAMIC) != 0
        assert sc["n"] == n and int((~dyn).sum()) == statics, k
        # SceneManager::load_scene: inverse mass 1 / mass, statics all zero (scene_manager.hpp:855-856)
        assert np.allclose(sc["inv_mass"][dyn], 1.0 / sc["mass"][dyn])
        assert (sc["inv_mass"][~dyn] == 0).all() and (sc["inv_inertia"][~dyn] == 0).all()


def test_box_pool_layout_follows_the_reference_hash():
    """scene_7's cube (ix, iy, iz) = (2, 5, 3): index-hashed jitter and tilt."""
    sc = io.load_reference_scene(7)
    ix, iy, iz = 2, 5, 3
    k = 6 + (iy * 6 + iz) * 6 + ix
    h1, h2, h3 = ix * 3 + iy * 5 + iz * 7, ix * 7 + iy * 3 + iz * 5, ix * 5 + iy * 7 + iz * 3
    x = -3.0 + 1.2 * ix + (h1 % 11 - 5.0) * 0.05
    y = 12.0 + 2.8 * iy + (h3 % 11 - 5.0) * 0.20
    z = 11.0 + 1.2 * iz + (h2 % 11 - 5.0) * 0.05
    assert np.allclose(sc["pos"][k], [x, y, z], atol=1e-5)
    phi, ang = (h3 % 16) * 0.3927, 0.07 + (h1 % 7) * 0.025
    sh = math.sin(0.5 * ang)
    assert np.allclose(sc["quat"][k], [math.cos(phi) * sh, 0.0, math.sin(phi) * sh, math.cos(0.5 * ang)], atol=1e-6)
    assert np.allclose(sc["half"][6:], 0.5) and np.allclose(sc["mass"][6:], 5.0)


def test_ramp_scene_friction_pairs():
    """scene_4: cube frictions 0.04 / 0.25 / 1.0 against friction-1 ramps (effective 0.2 / 0.5 / 1)."""
    sc = io.load_reference_scene(4)
    assert sorted(set(np.round(sc["friction"][4:].astype(np.float64), 4).tolist())) == [0.04, 0.25, 1.0]
    assert np.allclose(sc["friction"][:4], 1.0)


def test_voxel_scene_round_trips_through_a_file(tmp_path):
    sc = io.load_reference_scene(5)
    assert len(sc["voxel_shapes"]) == 3 and (sc["shape"] == scenes.SHAPE_VOXEL).sum() == 9
    path = str(tmp_path / "s5.npz")
    io.save_scene(sc, path)
    back = io.load_scene(path)
    for key in io._ARRAYS + io._OPTIONAL:
        assert np.array_equal(back[key], sc[key]), key
