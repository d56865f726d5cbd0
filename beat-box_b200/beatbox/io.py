"""Scene description and world-state files (numpy .npz).

A scene is the dict `beatbox.scenes` builds (per-body arrays plus "n" and an optional Morton box
"bounds"); the reference describes its scenes in code instead (src/scene_manager.hpp:114-823).
A checkpoint is a scene whose poses, velocities and flags are a world's current state, so
`World.add_scene` (or `world_from_scene`) restores it.  Persistent contacts are not stored: a
restored world restarts its warm start, as a scene load does in the reference.
"""
from __future__ import annotations

import numpy as np

_ARRAYS = ("pos", "quat", "half", "shape", "flags", "mass", "inv_mass", "inv_inertia", "friction", "restitution",
           "vel", "omega")


def save_scene(scene: dict, path: str) -> None:
    data = {k: np.asarray(scene[k]) for k in _ARRAYS}
    data["n"] = np.asarray(int(scene["n"]))
    b = scene.get("bounds")
    if b is not None:
        data["bounds"] = np.asarray([b[0], b[1]], np.float32)
    np.savez_compressed(path, **data)


def load_scene(path: str) -> dict:
    with np.load(path) as z:
        scene = {k: np.ascontiguousarray(z[k]) for k in _ARRAYS}
        scene["n"] = int(z["n"])
        scene["bounds"] = (z["bounds"][0].tolist(), z["bounds"][1].tolist()) if "bounds" in z.files else None
    return scene


def checkpoint(world, scene: dict) -> dict:
    """The scene with `world`'s current state (poses, velocities, sleep flags)."""
    st = world.read_state()
    out = dict(scene)
    out["pos"], out["quat"], out["vel"], out["omega"] = st["pos"], st["quat"], st["vel"], st["omega"]
    out["flags"] = world.read_flags().astype(np.uint32)
    return out
