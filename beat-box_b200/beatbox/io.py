"""Scene description and world-state files (numpy .npz).

A scene is the dict `beatbox.scenes` builds (per-body arrays plus "n", an optional Morton box
"bounds" and, for concave bodies, "voxel_shapes"); the reference describes its scenes in code
instead (src/scene_manager.hpp:114-823).  Its seven demo scenes ship as data files in
``beatbox/scene_data`` (``load_reference_scene``).

A checkpoint holds the scene, the solver parameters and the world's state image
(``World.save_state``: poses, velocities, sleep timers and the persistent contacts with their
impulses, anchors and warm-start counters), so ``restore_world`` gives a world that steps
bit for bit as the saved one would have.  The image is the world's device footprint in size.
``checkpoint`` alone gives the scene with the current poses, velocities and flags (a cold
restart: warm starts begin again, as a scene load does in the reference).
"""
from __future__ import annotations

import os

import numpy as np

_ARRAYS = ("pos", "quat", "half", "shape", "flags", "mass", "inv_mass", "inv_inertia", "friction", "restitution",
           "vel", "omega")
_OPTIONAL = ("inv_inertia_off", "voxel")
SCENE_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scene_data")


def _scene_arrays(scene: dict) -> dict:
    data = {k: np.asarray(scene[k]) for k in _ARRAYS}
    for k in _OPTIONAL:
        if k in scene:
            data[k] = np.asarray(scene[k])
    data["n"] = np.asarray(int(scene["n"]))
    b = scene.get("bounds")
    if b is not None:
        data["bounds"] = np.asarray([b[0], b[1]], np.float32)
    for i, v in enumerate(scene.get("voxel_shapes", [])):
        data[f"voxel_solid_{i}"] = np.asarray(v["solid"], np.uint8)
        data[f"voxel_size_{i}"] = np.asarray(float(v["voxel_size"]), np.float64)
    return data


def _scene_from(z) -> dict:
    scene = {k: np.ascontiguousarray(z[k]) for k in _ARRAYS}
    for k in _OPTIONAL:
        if k in z.files:
            scene[k] = np.ascontiguousarray(z[k])
    scene["n"] = int(z["n"])
    scene["bounds"] = (z["bounds"][0].tolist(), z["bounds"][1].tolist()) if "bounds" in z.files else None
    shapes = []
    while f"voxel_solid_{len(shapes)}" in z.files:
        i = len(shapes)
        shapes.append({"solid": np.ascontiguousarray(z[f"voxel_solid_{i}"]),
                       "voxel_size": float(z[f"voxel_size_{i}"])})
    if shapes:
        scene["voxel_shapes"] = shapes
    return scene


def save_scene(scene: dict, path: str) -> None:
    np.savez_compressed(path, **_scene_arrays(scene))


def load_scene(path: str) -> dict:
    with np.load(path) as z:
        return _scene_from(z)


def load_reference_scene(k: int) -> dict:
    """The reference's scene k (1..7, src/scene_manager.hpp:114-823) from the shipped data files."""
    path = os.path.join(SCENE_DATA, f"scene_{k}.npz")
    if not os.path.exists(path):
        raise ValueError(f"no data file for reference scene {k} (the reference has scenes 1..7)")
    return load_scene(path)


def checkpoint(world, scene: dict) -> dict:
    """The scene with `world`'s current state (poses, velocities, sleep flags)."""
    st = world.read_state()
    out = dict(scene)
    out["pos"], out["quat"], out["vel"], out["omega"] = st["pos"], st["quat"], st["vel"], st["omega"]
    out["flags"] = world.read_flags().astype(np.uint32)
    return out


def save_checkpoint(world, scene: dict, path: str, max_bodies: int | None = None, pairs_per_body: int = 16) -> None:
    """The scene the world was built from (its bodies added with World.add_scene, in order), the
    world's capacity and solver parameters, and its state image."""
    data = _scene_arrays(scene)
    data["state"] = world.save_state()
    data["params"] = np.frombuffer(bytes(world.params), np.uint8)
    data["capacity"] = np.asarray([int(max_bodies or scene["n"]), int(pairs_per_body)], np.int64)
    np.savez_compressed(path, **data)


def restore_world(path: str, device: int = -1):
    """A world built from a checkpoint: created with the saved capacity, the scene's bodies added,
    the parameters set and the state image loaded.  Returns (world, scene)."""
    from . import SolverParams, World

    with np.load(path) as z:
        scene = _scene_from(z)
        cap, ppb = (int(v) for v in z["capacity"])
        p = SolverParams.from_buffer_copy(z["params"].tobytes())
        state = np.ascontiguousarray(z["state"])
    w = World(cap, pairs_per_body=ppb, device=device)
    w.add_scene(scene)
    w.set_params(p)
    w.load_state(state)
    return w, scene


__all__ = ["save_scene", "load_scene", "load_reference_scene", "checkpoint", "save_checkpoint", "restore_world",
           "SCENE_DATA"]
