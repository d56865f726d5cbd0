"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the oracle (oracle/liboracle.so).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.  The oracle
is a CPU restatement of the reference step (see bb_oracle.hpp); it is the checker, never the
thing measured as the product.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


class SolverParams(ctypes.Structure):
    _fields_ = [
        ("solver", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("quirks", ctypes.c_uint32),
        ("iterations", ctypes.c_uint32), ("relax_iterations", ctypes.c_uint32), ("gc_rounds", ctypes.c_uint32),
        ("gravity", ctypes.c_float), ("linear_damping", ctypes.c_float), ("angular_damping", ctypes.c_float),
        ("contact_hertz", ctypes.c_float), ("penetration_cap", ctypes.c_float),
        ("sleep_lin_vel2", ctypes.c_float), ("sleep_ang_vel2", ctypes.c_float), ("sleep_steps", ctypes.c_uint32),
        ("avbd_iterations", ctypes.c_uint32), ("avbd_beta", ctypes.c_float), ("avbd_gamma", ctypes.c_float),
        ("avbd_k_min", ctypes.c_float), ("avbd_k_max", ctypes.c_float), ("avbd_margin", ctypes.c_float),
        ("avbd_stick_thresh", ctypes.c_float), ("avbd_stick_slop", ctypes.c_float),
        ("avbd_color_rounds", ctypes.c_uint32), ("avbd_shock_layers", ctypes.c_uint32),
        ("avbd_post_stab_sweeps", ctypes.c_uint32), ("schedule", ctypes.c_uint32), ("broad_threads", ctypes.c_uint32),
        ("narrow_blocks_per_sm", ctypes.c_uint32), ("pgs_stage_next", ctypes.c_uint32), ("bounds_mode", ctypes.c_uint32),
        ("world_min", ctypes.c_float * 3), ("world_extent", ctypes.c_float * 3),
    ]


class StepStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "body_count", "active_body_count", "pair_count", "manifold_count", "contact_count", "island_count",
        "graph_color_count", "graph_color_overflow", "graph_color_violations", "avbd_color_count",
        "avbd_violations", "sleeping_count", "fresh_contacts", "stick_count")] + [
        ("max_penetration", ctypes.c_float), ("error_flags", ctypes.c_uint32), ("pair_capacity", ctypes.c_uint32),
        ("substeps_run", ctypes.c_uint32), ("solved_manifolds", ctypes.c_uint32), ("solved_contacts", ctypes.c_uint32),
        ("graph_color_rounds", ctypes.c_uint32), ("error_site", ctypes.c_uint32)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ only)."""
    if force or not os.path.exists(LIB_PATH) or _stale():
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return LIB_PATH


def _stale() -> bool:
    t = os.path.getmtime(LIB_PATH)
    for f in ("bb_oracle.cpp", "bb_oracle.hpp", "bb_oracle_world.hpp", "bb_oracle_math.hpp"):
        if os.path.getmtime(os.path.join(HERE, f)) > t:
            return True
    return os.path.getmtime(os.path.join(HERE, "..", "include", "beatbox.h")) > t


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.c_uint32] + [P] * 12 + [ctypes.c_int, ctypes.c_int]
        L.orc_destroy.argtypes = [P]
        L.orc_default_params.argtypes = [ctypes.POINTER(SolverParams)]
        L.orc_set_params.argtypes = [P, ctypes.POINTER(SolverParams)]
        L.orc_step.argtypes = [P, ctypes.c_float, ctypes.c_uint32]
        L.orc_collide.argtypes = [P, ctypes.c_uint32]
        L.orc_skip_warm_starting_once.argtypes = [P]
        L.orc_inject_manifolds.argtypes = [P, P, P, ctypes.c_uint32]
        L.orc_set_carry_frozen.argtypes = [P, ctypes.c_int]
        L.orc_read_state.argtypes = [P, P, P, P, P, P]
        L.orc_read_stats.argtypes = [P, ctypes.POINTER(StepStats)]
        L.orc_debug_read.restype = ctypes.c_uint64
        L.orc_debug_read.argtypes = [P, ctypes.c_uint32, P, ctypes.c_uint64]
        L.orc_morton.restype = ctypes.c_uint32
        L.orc_morton.argtypes = [P, P, P]
        L.orc_leaf_aabb.argtypes = [ctypes.c_uint32, P, P, P, P]
        L.orc_add_voxel_shape.restype = ctypes.c_uint32
        L.orc_add_voxel_shape.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, P]
        L.orc_set_voxel_bodies.argtypes = [P, P, P]
        L.orc_voxel_shape.argtypes = [P, ctypes.c_uint32, P, P, P]
        L.orc_collide_pair.restype = ctypes.c_int
        L.orc_collide_pair.argtypes = [ctypes.c_uint32, P, P, P, ctypes.c_uint32, P, P, P, ctypes.c_int, P, P, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def default_params() -> SolverParams:
    p = SolverParams()
    lib().orc_default_params(ctypes.byref(p))
    return p


class Oracle:
    """One oracle world built from a scene dict (see beatbox.scenes)."""

    def __init__(self, scene: dict, double: bool = True, threads: int = 1, params: SolverParams | None = None):
        self._keep = {}
        L = lib()
        n = int(scene["n"])
        arr = {}
        for k, dt in (("pos", np.float32), ("quat", np.float32), ("vel", np.float32), ("omega", np.float32),
                      ("shape", np.uint32), ("half", np.float32), ("flags", np.uint32), ("mass", np.float32),
                      ("inv_mass", np.float32), ("inv_inertia", np.float32), ("friction", np.float32),
                      ("restitution", np.float32)):
            arr[k] = np.ascontiguousarray(scene[k], dtype=dt)
        self.n = n
        self.h = L.orc_create(n, _ptr(arr["pos"]), _ptr(arr["quat"]), _ptr(arr["vel"]), _ptr(arr["omega"]),
                              _ptr(arr["shape"]), _ptr(arr["half"]), _ptr(arr["flags"]), _ptr(arr["mass"]),
                              _ptr(arr["inv_mass"]), _ptr(arr["inv_inertia"]), _ptr(arr["friction"]),
                              _ptr(arr["restitution"]), 1 if double else 0, int(threads))
        if scene.get("voxel_shapes") or "inv_inertia_off" in scene:
            for v in scene.get("voxel_shapes", []):
                g = np.ascontiguousarray(np.asarray(v["solid"]) != 0, dtype=np.uint8)
                nz, ny, nx = g.shape
                L.orc_add_voxel_shape(self.h, nx, ny, nz, float(v["voxel_size"]), _ptr(g))
            vidx = np.ascontiguousarray(scene.get("voxel", np.zeros(n)), dtype=np.uint32)
            off = np.ascontiguousarray(scene.get("inv_inertia_off", np.zeros((n, 3))), dtype=np.float32)
            L.orc_set_voxel_bodies(self.h, _ptr(vidx), _ptr(off))
        if params is not None:
            self.set_params(params)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_params(self, p: SolverParams):
        lib().orc_set_params(self.h, ctypes.byref(p))

    def step(self, dt: float, substeps: int = 1):
        lib().orc_step(self.h, ctypes.c_float(dt), substeps)

    def collide(self, stage: int):
        lib().orc_collide(self.h, stage)

    def set_carry_frozen(self, on: bool):
        lib().orc_set_carry_frozen(self.h, 1 if on else 0)

    def skip_warm_starting_once(self):
        lib().orc_skip_warm_starting_once(self.h)

    def inject_manifolds(self, manifolds: np.ndarray, contacts: np.ndarray):
        """The next substep's narrow phase takes this geometry (records in the library's
        bb_manifold_info / bb_contact_info layouts, 8 contacts per manifold) instead of its own."""
        m = np.ascontiguousarray(manifolds)
        c = np.ascontiguousarray(contacts)
        assert c.size == 8 * m.size
        self._keep["inj"] = (m, c)
        lib().orc_inject_manifolds(self.h, _ptr(m), _ptr(c), int(m.size))

    def state(self):
        pos = np.zeros((self.n, 3))
        quat = np.zeros((self.n, 4))
        vel = np.zeros((self.n, 3))
        om = np.zeros((self.n, 3))
        flags = np.zeros(self.n, np.uint32)
        lib().orc_read_state(self.h, _ptr(pos), _ptr(quat), _ptr(vel), _ptr(om), _ptr(flags))
        return dict(pos=pos, quat=quat, vel=vel, omega=om, flags=flags)

    def stats(self) -> dict:
        s = StepStats()
        lib().orc_read_stats(self.h, ctypes.byref(s))
        return s.as_dict()

    def debug_read(self, which: int, dtype=np.uint32, cap: int = 1 << 26):
        buf = np.empty(cap, np.uint8)
        cnt = lib().orc_debug_read(self.h, which, _ptr(buf), buf.nbytes)
        return cnt, buf


def voxel_shape(o: "Oracle", index: int) -> dict:
    """The oracle's own build of a voxel shape: origin, box, counts and surface list."""
    f9 = np.zeros(9, np.float32)
    u2 = np.zeros(2, np.uint32)
    lib().orc_voxel_shape(o.h, index, _ptr(f9), _ptr(u2), None)
    surf = np.zeros(int(u2[1]), np.uint32)
    lib().orc_voxel_shape(o.h, index, _ptr(f9), _ptr(u2), _ptr(surf))
    return {"grid_origin": f9[:3], "box_min": f9[3:6], "box_max": f9[6:], "solid_count": int(u2[0]),
            "surface_count": int(u2[1]), "surface": surf}


def morton(p, wmin, wext) -> int:
    p = np.ascontiguousarray(p, np.float32)
    wmin = np.ascontiguousarray(wmin, np.float32)
    wext = np.ascontiguousarray(wext, np.float32)
    return int(lib().orc_morton(_ptr(p), _ptr(wmin), _ptr(wext)))


def leaf_aabb(shape, half, p, q) -> np.ndarray:
    out = np.zeros(6, np.float32)
    half = np.ascontiguousarray(half, np.float32)
    p = np.ascontiguousarray(p, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    lib().orc_leaf_aabb(int(shape), _ptr(half), _ptr(p), _ptr(q), _ptr(out))
    return out


def collide_pair(shape_a, half_a, pos_a, quat_a, shape_b, half_b, pos_b, quat_b, sat_frame_quirk=True):
    """Narrow phase of one pair in FP64: (count, normal, key, positions[count,3], depths[count])."""
    f = lambda a, t: np.ascontiguousarray(a, t)  # noqa: E731
    ha, hb = f(half_a, np.float32), f(half_b, np.float32)
    pa, pb, qa, qb = f(pos_a, np.float64), f(pos_b, np.float64), f(quat_a, np.float64), f(quat_b, np.float64)
    normal = np.zeros(3)
    key = ctypes.c_int(0)
    pos = np.zeros((8, 3))
    dep = np.zeros(8)
    n = lib().orc_collide_pair(int(shape_a), _ptr(ha), _ptr(pa), _ptr(qa), int(shape_b), _ptr(hb), _ptr(pb), _ptr(qb),
                               1 if sat_frame_quirk else 0, _ptr(normal), ctypes.byref(key), _ptr(pos), _ptr(dep))
    return n, normal, key.value, pos[:n], dep[:n]
