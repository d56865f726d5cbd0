"""beatbox -- Python host side of the B200 rigid-body step library (libbeatbox.so).

``World`` wraps the C ABI of include/beatbox.h with numpy arrays.  ``RigidBodyManager`` mirrors
the reference's class of that name (src/rigid_body_manager.hpp:12-70): create / simulate /
read_back_sim_config / set_sim_flags / clear_sim_flags / set_sim_type /
skip_warm_starting_once, so code written against the reference's manager reads the same.

The library is CUDA-only: importing works anywhere, but creating a world needs the built
libbeatbox.so and a GPU, and fails loudly otherwise (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import scenes  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libbeatbox.so")

# status codes and flags (include/beatbox.h)
OK, E_INVALID, E_CAPACITY, E_CUDA, E_DEVICE_LIMIT, E_BUDGET, E_UNSUPPORTED = range(7)
BODY_DYNAMIC, BODY_GRAVITY, BODY_SLEEPING = 1 << 1, 1 << 2, 1 << 3
SHAPE_BOX, SHAPE_SPHERE, SHAPE_VOXEL = 0, 1, 2
INERTIA_PHYSICAL, INERTIA_REFERENCE, INERTIA_EXPLICIT = 0, 1, 2
SOLVER_PGS, SOLVER_PGS_SOFT, SOLVER_AVBD = 0, 1, 2
SIM_ACCUM_IMPULSE, SIM_FRICTION, SIM_WARM_STARTING, SIM_ADVECTION = 1, 2, 4, 8
SIM_DEBUG_INFO, SIM_USE_GRAPH_COLORING, SIM_SLEEPING_ENABLED = 16, 32, 128
SIM_DEFAULT_FLAGS = SIM_ACCUM_IMPULSE | SIM_FRICTION | SIM_WARM_STARTING | SIM_ADVECTION | SIM_DEBUG_INFO | \
    SIM_USE_GRAPH_COLORING | SIM_SLEEPING_ENABLED
QUIRK_GRAVITY_IMPULSE, QUIRK_SAT_FRAME, QUIRK_INERTIA_TRANSPOSE = 1, 2, 4
QUIRKS_REFERENCE, QUIRKS_PHYSICAL = 7, 0
BOUNDS_FIXED, BOUNDS_AUTO = 0, 1
SCHEDULE_DATAFLOW, SCHEDULE_COLOUR_BARRIER = 0, 1
SORT_STATIC_MAX_KEYS = 262144
EDGE_COLOR_OVERFLOW = 0xFFFFFFFF
EDGE_COLOR_RESTING = 0xFFFFFFFE  # the manifold's island has no awake body: not coloured, not solved
DBG = dict(morton=1, sorted_keys=2, sorted_ids=3, lbvh_child=4, leaf_aabb=5, node_aabb=6, pairs=7,
           manifolds=8, contacts=9, edge_colors=10, body_colors=11, islands=12, support_depth=13, body_inertia=14)


class BeatboxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"beatbox error {code}: {msg}")
        self.code = code


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


class WorldDesc(ctypes.Structure):
    _fields_ = [("max_bodies", ctypes.c_uint32), ("pairs_per_body", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("stream", ctypes.c_void_p)]


class BodyDesc(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("rotation", ctypes.c_float * 4), ("velocity", ctypes.c_float * 3),
                ("omega", ctypes.c_float * 3), ("shape", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("mass", ctypes.c_float), ("density", ctypes.c_float), ("friction", ctypes.c_float),
                ("restitution", ctypes.c_float), ("inertia_mode", ctypes.c_uint32), ("inv_inertia", ctypes.c_float * 3),
                ("inv_inertia_off", ctypes.c_float * 3)]


class VoxelInfo(ctypes.Structure):
    _fields_ = [("grid_origin", ctypes.c_float * 3), ("box_min", ctypes.c_float * 3), ("box_max", ctypes.c_float * 3),
                ("solid_count", ctypes.c_uint32), ("surface_count", ctypes.c_uint32), ("unit_mass", ctypes.c_float),
                ("unit_inv_inertia", ctypes.c_float * 6)]


BODY_DTYPE = np.dtype([("position", "<f4", 3), ("rotation", "<f4", 4), ("velocity", "<f4", 3), ("omega", "<f4", 3),
                       ("shape", "<u4"), ("flags", "<u4"), ("mass", "<f4"), ("density", "<f4"),
                       ("friction", "<f4"), ("restitution", "<f4"), ("inertia_mode", "<u4"),
                       ("inv_inertia", "<f4", 3), ("inv_inertia_off", "<f4", 3)])
assert BODY_DTYPE.itemsize == ctypes.sizeof(BodyDesc)


class BatchWorldDesc(ctypes.Structure):
    _fields_ = [("world_min", ctypes.c_float * 3), ("world_extent", ctypes.c_float * 3)]


class ShapeDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("half", ctypes.c_float * 3)]


class ServerDesc(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_active", ctypes.c_uint32),
                ("pairs_per_body", ctypes.c_uint32), ("device", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("world", ctypes.c_uint64), ("shapes", ctypes.POINTER(ShapeDesc)), ("n_shapes", ctypes.c_uint32),
                ("bodies", ctypes.POINTER(BodyDesc)), ("n_bodies", ctypes.c_uint32),
                ("world_min", ctypes.c_float * 3), ("world_extent", ctypes.c_float * 3),
                ("params", SolverParams), ("dt", ctypes.c_float), ("substeps", ctypes.c_uint32),
                ("steps", ctypes.c_uint32)]


class RequestStatus(ctypes.Structure):
    _fields_ = [("done", ctypes.c_uint32), ("result", ctypes.c_int32), ("submit_s", ctypes.c_double),
                ("start_s", ctypes.c_double), ("finish_s", ctypes.c_double), ("error_flags", ctypes.c_uint32),
                ("error_site", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("body_steps", ctypes.c_uint64), ("evictions", ctypes.c_uint64), ("worlds_created", ctypes.c_uint64),
                ("resident_bytes", ctypes.c_uint64), ("active", ctypes.c_uint32), ("queued", ctypes.c_uint32),
                ("resident_worlds", ctypes.c_uint32), ("known_worlds", ctypes.c_uint32),
                ("materialise_s", ctypes.c_double), ("issue_s", ctypes.c_double), ("batch_steps", ctypes.c_uint64),
                ("slot_steps", ctypes.c_uint64)]


class StepStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "body_count", "active_body_count", "pair_count", "manifold_count", "contact_count", "island_count",
        "graph_color_count", "graph_color_overflow", "graph_color_violations", "avbd_color_count",
        "avbd_violations", "sleeping_count", "fresh_contacts", "stick_count")] + [
        ("max_penetration", ctypes.c_float), ("error_flags", ctypes.c_uint32), ("pair_capacity", ctypes.c_uint32),
        ("substeps_run", ctypes.c_uint32), ("solved_manifolds", ctypes.c_uint32),
        ("solved_contacts", ctypes.c_uint32), ("graph_color_rounds", ctypes.c_uint32), ("error_site", ctypes.c_uint32)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


MANIFOLD_DTYPE = np.dtype([("body_a", "<u4"), ("body_b", "<u4"), ("key", "<i4"), ("contact_count", "<i4"),
                           ("normal", "<f4", 3), ("color", "<u4"), ("tangent", "<f4", (2, 3))])
CONTACT_DTYPE = np.dtype([("position", "<f4", 3), ("penetration", "<f4"), ("normal_impulse", "<f4"),
                          ("tangent_impulse", "<f4", 2), ("feature", "<u4"), ("warm_start", "<u4"),
                          ("penalty", "<f4")])

# exported symbols of include/beatbox.h: name -> (restype, argtypes)
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_SIG = {
    "bb_default_solver_params": (None, [ctypes.POINTER(SolverParams)]),
    "bb_world_create": (ctypes.c_int32, [ctypes.POINTER(WorldDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "bb_world_destroy": (ctypes.c_int32, [_P]),
    "bb_add_box_shape": (ctypes.c_int32, [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.POINTER(_U32)]),
    "bb_add_sphere_shape": (ctypes.c_int32, [_P, ctypes.c_float, ctypes.POINTER(_U32)]),
    "bb_add_voxel_shape": (ctypes.c_int32, [_P, _U32, _U32, _U32, ctypes.c_float, _P, ctypes.POINTER(_U32)]),
    "bb_voxel_shape_info": (ctypes.c_int32, [_U32, _U32, _U32, ctypes.c_float, _P, ctypes.POINTER(VoxelInfo), _P, _U32]),
    "bb_add_bodies": (ctypes.c_int32, [_P, ctypes.POINTER(BodyDesc), _U32, ctypes.POINTER(_U32)]),
    "bb_add_world": (ctypes.c_int32, [_P, ctypes.POINTER(BatchWorldDesc), ctypes.POINTER(BodyDesc), _U32,
                                      ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "bb_world_count": (_U32, [_P]),
    "bb_world_pause": (ctypes.c_int32, [_P, _U32, _U32]),
    "bb_world_refill": (ctypes.c_int32, [_P, _U32, ctypes.POINTER(BatchWorldDesc), ctypes.POINTER(BodyDesc), _U32]),
    "bb_set_material": (ctypes.c_int32, [_P, _U32, _U32, ctypes.c_float, ctypes.c_float]),
    "bb_set_solver_params": (ctypes.c_int32, [_P, ctypes.POINTER(SolverParams)]),
    "bb_get_solver_params": (ctypes.c_int32, [_P, ctypes.POINTER(SolverParams)]),
    "bb_step": (ctypes.c_int32, [_P, ctypes.c_float, _U32]),
    "bb_sync": (ctypes.c_int32, [_P]),
    "bb_read_state": (ctypes.c_int32, [_P, _P, _P, _P, _P]),
    "bb_write_state": (ctypes.c_int32, [_P, _P, _P, _P, _P]),
    "bb_read_flags": (ctypes.c_int32, [_P, _P]),
    "bb_body_count": (_U32, [_P]),
    "bb_read_stats": (ctypes.c_int32, [_P, ctypes.POINTER(StepStats)]),
    "bb_skip_warm_starting_once": (ctypes.c_int32, [_P]),
    "bb_debug_collide": (ctypes.c_int32, [_P, _U32]),
    "bb_debug_read": (ctypes.c_int32, [_P, _U32, _P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "bb_debug_wait_limit": (ctypes.c_int32, [_P, _U32, _U32]),
    "bb_world_stream": (ctypes.c_void_p, [_P]),
    "bb_set_profiling": (ctypes.c_int32, [_P, ctypes.c_int32]),
    "bb_read_stage_times": (ctypes.c_int32, [_P, _P, _U32, ctypes.POINTER(_U32), _P, _U32]),
    "bb_kernel_launch_count": (ctypes.c_uint64, [_P]),
    "bb_radix_sort_pairs": (ctypes.c_int32, [_P, _P, _P, _P, _U32, _U32, _P]),
    "bb_radix_sort_pairs_static": (ctypes.c_int32, [_P, _P, _P, _P, _U32, _U32, _P]),
    "bb_radix_sort_error_flags": (ctypes.c_int32, [_U32, _P, ctypes.POINTER(_U32)]),
    "bb_autotune": (ctypes.c_int32, [_P, ctypes.c_float, _U32, _U32, ctypes.POINTER(SolverParams)]),
    "bb_update_transforms": (ctypes.c_int32, [_P]),
    "bb_transforms_device": (ctypes.c_void_p, [_P]),
    "bb_read_transforms": (ctypes.c_int32, [_P, _P]),
    "bb_read_contact_points": (ctypes.c_int32, [_P, _P, _U32, ctypes.POINTER(_U32)]),
    "bb_world_device_bytes": (ctypes.c_uint64, [_P]),
    "bb_world_clear": (ctypes.c_int32, [_P]),
    "bb_world_save_state": (ctypes.c_int32, [_P, _P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "bb_world_set_auto_regrow": (ctypes.c_int32, [_P, _U32]),
    "bb_world_load_state": (ctypes.c_int32, [_P, _P, ctypes.c_uint64]),
    "bb_world_bytes_for": (ctypes.c_uint64, [_U32, _U32]),
    "bb_server_create": (ctypes.c_int32, [ctypes.POINTER(ServerDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "bb_server_destroy": (ctypes.c_int32, [_P]),
    "bb_server_submit": (ctypes.c_int32, [_P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]),
    "bb_server_poll": (ctypes.c_int32, [_P, ctypes.c_uint64, ctypes.POINTER(RequestStatus)]),
    "bb_server_wait": (ctypes.c_int32, [_P, ctypes.c_uint64, ctypes.POINTER(RequestStatus)]),
    "bb_server_read_state": (ctypes.c_int32, [_P, ctypes.c_uint64, _P, _P, _P, _P, ctypes.POINTER(_U32)]),
    "bb_server_get_stats": (ctypes.c_int32, [_P, ctypes.POINTER(ServerStats)]),
    "bb_last_error_string": (ctypes.c_char_p, []),
    "bb_version": (ctypes.c_char_p, []),
}

_lib = None


def load_library(path: str | None = None):
    """Load libbeatbox.so (building it first if it is missing and nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_bb_build", os.path.join(PKG, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = ctypes.CDLL(path)
    for name, (res, args) in _SIG.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(code: int):
    if code != OK:
        raise BeatboxError(code, _lib.bb_last_error_string().decode())


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def default_params() -> SolverParams:
    p = SolverParams()
    load_library().bb_default_solver_params(ctypes.byref(p))
    return p


def make_params(**kw) -> SolverParams:
    p = default_params()
    for k, v in kw.items():
        if k in ("world_min", "world_extent"):
            getattr(p, k)[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


class World:
    """One simulated world on the GPU (wraps bb_world_*)."""

    def __init__(self, max_bodies: int, pairs_per_body: int = 16, device: int = -1, stream: int | None = None):
        L = load_library()
        desc = WorldDesc(max_bodies, pairs_per_body, device, stream)
        h = ctypes.c_void_p()
        _check(L.bb_world_create(ctypes.byref(desc), ctypes.byref(h)))
        self.h = h
        self.L = L
        self._shape_cache: dict = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.bb_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- construction --------------------------------------------------------------------
    def add_box_shape(self, hx: float, hy: float, hz: float) -> int:
        out = _U32()
        _check(self.L.bb_add_box_shape(self.h, hx, hy, hz, ctypes.byref(out)))
        return out.value

    def add_sphere_shape(self, r: float) -> int:
        out = _U32()
        _check(self.L.bb_add_sphere_shape(self.h, r, ctypes.byref(out)))
        return out.value

    def add_voxel_shape(self, solid, voxel_size: float) -> int:
        """Voxel shape from an occupancy grid indexed solid[z, y, x] (non-zero = solid)."""
        g = np.ascontiguousarray(np.asarray(solid) != 0, dtype=np.uint8)
        nz, ny, nx = g.shape
        out = _U32()
        _check(self.L.bb_add_voxel_shape(self.h, nx, ny, nz, float(voxel_size), g.ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(out)))
        return out.value

    def _shape_for(self, shape: int, half) -> int:
        key = (int(shape), float(half[0]), float(half[1]), float(half[2]))
        h = self._shape_cache.get(key)
        if h is None:
            h = self.add_box_shape(*key[1:]) if shape == SHAPE_BOX else self.add_sphere_shape(key[1])
            self._shape_cache[key] = h
        return h

    def _scene_descs(self, scene: dict, inertia_mode: int):
        """bb_body_desc array of a scene, filled column-wise through a numpy view."""
        n = int(scene["n"])
        descs = (BodyDesc * n)()
        a = np.frombuffer(descs, dtype=BODY_DTYPE, count=n)
        a["position"] = scene["pos"]
        a["rotation"] = scene["quat"]
        a["velocity"] = scene["vel"]
        a["omega"] = scene["omega"]
        vox_handles = [self.add_voxel_shape(v["solid"], v["voxel_size"]) for v in scene.get("voxel_shapes", [])]
        vidx = scene.get("voxel")
        a["shape"] = [vox_handles[int(vidx[i])] if int(t) == SHAPE_VOXEL else self._shape_for(int(t), h)
                      for i, (t, h) in enumerate(zip(scene["shape"].tolist(), scene["half"].tolist()))]
        a["flags"] = scene["flags"]
        a["mass"] = scene["mass"]
        a["density"] = 0.0
        a["friction"] = scene["friction"]
        a["restitution"] = scene["restitution"]
        a["inertia_mode"] = inertia_mode
        a["inv_inertia"] = scene["inv_inertia"]
        if "inv_inertia_off" in scene:
            a["inv_inertia_off"] = scene["inv_inertia_off"]
        return descs, n

    def add_scene(self, scene: dict, inertia_mode: int = INERTIA_EXPLICIT) -> int:
        """Add every body of a beatbox.scenes dict; masses and inverse inertias are taken from
        the scene (the oracle gets the same arrays)."""
        descs, n = self._scene_descs(scene, inertia_mode)
        first = _U32()
        _check(self.L.bb_add_bodies(self.h, descs, n, ctypes.byref(first)))
        return first.value

    def add_world(self, scene: dict, world_min, world_extent, inertia_mode: int = INERTIA_EXPLICIT):
        """Append a scene as an independent world of a batch (bodies of different worlds
        never collide).  Returns (world index, first body id)."""
        descs, n = self._scene_descs(scene, inertia_mode)
        wd = BatchWorldDesc()
        wd.world_min[:] = [float(v) for v in world_min]
        wd.world_extent[:] = [float(v) for v in world_extent]
        wi, first = _U32(), _U32()
        _check(self.L.bb_add_world(self.h, ctypes.byref(wd), descs, n, ctypes.byref(wi), ctypes.byref(first)))
        return wi.value, first.value

    def pause_world(self, index: int, paused: bool = True):
        """Pause (or resume) world `index` of a batch: while paused it is left exactly as it is."""
        _check(self.L.bb_world_pause(self.h, index, 1 if paused else 0))

    def refill_world(self, index: int, scene: dict, world_min, world_extent, inertia_mode: int = INERTIA_EXPLICIT):
        """Replace the bodies of world `index`'s slot by a new scene (at most the slot's size)."""
        descs, n = self._scene_descs(scene, inertia_mode)
        wd = BatchWorldDesc()
        wd.world_min[:] = [float(v) for v in world_min]
        wd.world_extent[:] = [float(v) for v in world_extent]
        _check(self.L.bb_world_refill(self.h, index, ctypes.byref(wd), descs, n))

    @property
    def n_worlds(self) -> int:
        return int(self.L.bb_world_count(self.h))

    def add_bodies(self, descs) -> int:
        arr = (BodyDesc * len(descs))(*descs)
        first = _U32()
        _check(self.L.bb_add_bodies(self.h, arr, len(descs), ctypes.byref(first)))
        return first.value

    def set_material(self, first: int, n: int, friction: float, restitution: float = 0.0):
        _check(self.L.bb_set_material(self.h, first, n, friction, restitution))

    # ---- parameters --------------------------------------------------------------------
    @property
    def params(self) -> SolverParams:
        p = SolverParams()
        _check(self.L.bb_get_solver_params(self.h, ctypes.byref(p)))
        return p

    def set_params(self, p: SolverParams | None = None, **kw):
        p = p if p is not None else self.params
        if not isinstance(p, SolverParams):  # a layout-identical struct (e.g. the oracle's)
            p = SolverParams.from_buffer_copy(bytes(p))
        for k, v in kw.items():
            if k in ("world_min", "world_extent"):
                getattr(p, k)[:] = [float(x) for x in v]
            else:
                setattr(p, k, v)
        _check(self.L.bb_set_solver_params(self.h, ctypes.byref(p)))

    # ---- stepping ------------------------------------------------------------------------
    def step(self, dt: float, substeps: int = 1):
        _check(self.L.bb_step(self.h, ctypes.c_float(dt), substeps))

    def autotune(self, dt: float, substeps: int = 1, trial_steps: int = 2) -> dict:
        """Time launch geometries / schedules on this world (each trial step advances it) and keep
        the fastest; returns the chosen tunables."""
        p = SolverParams()
        _check(self.L.bb_autotune(self.h, dt, substeps, trial_steps, ctypes.byref(p)))
        return dict(schedule=p.schedule, broad_threads=p.broad_threads, narrow_blocks_per_sm=p.narrow_blocks_per_sm,
                    pgs_stage_next=p.pgs_stage_next)

    def sync(self):
        _check(self.L.bb_sync(self.h))

    def skip_warm_starting_once(self):
        _check(self.L.bb_skip_warm_starting_once(self.h))

    @property
    def n(self) -> int:
        return int(self.L.bb_body_count(self.h))

    @property
    def stream(self) -> int:
        return self.L.bb_world_stream(self.h)

    def launches(self) -> int:
        return int(self.L.bb_kernel_launch_count(self.h))

    # ---- readback ------------------------------------------------------------------------
    def read_state(self, out: dict | None = None) -> dict:
        n = self.n
        out = out or dict(pos=np.empty((n, 3), np.float32), quat=np.empty((n, 4), np.float32),
                          vel=np.empty((n, 3), np.float32), omega=np.empty((n, 3), np.float32))
        _check(self.L.bb_read_state(self.h, _ptr(out["pos"]), _ptr(out["quat"]), _ptr(out["vel"]), _ptr(out["omega"])))
        return out

    def write_state(self, pos=None, quat=None, vel=None, omega=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)  # noqa: E731
        pos, quat, vel, omega = c(pos), c(quat), c(vel), c(omega)
        _check(self.L.bb_write_state(self.h, _ptr(pos), _ptr(quat), _ptr(vel), _ptr(omega)))

    def read_transforms(self) -> np.ndarray:
        """(n, 3, 4) affine transforms [R | t] of every body (world = R local + t)."""
        out = np.empty((self.n, 3, 4), np.float32)
        _check(self.L.bb_read_transforms(self.h, _ptr(out)))
        return out

    def read_contact_points(self) -> np.ndarray:
        """(k, 4) contact points of the last substep: position, depth."""
        cnt = _U32()
        _check(self.L.bb_read_contact_points(self.h, None, 0, ctypes.byref(cnt)))
        out = np.empty((cnt.value, 4), np.float32)
        _check(self.L.bb_read_contact_points(self.h, _ptr(out), cnt.value, ctypes.byref(cnt)))
        return out

    def read_flags(self) -> np.ndarray:
        f = np.empty(self.n, np.uint32)
        _check(self.L.bb_read_flags(self.h, _ptr(f)))
        return f

    def stats(self) -> dict:
        s = StepStats()
        _check(self.L.bb_read_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    def debug_collide(self, stage: int):
        _check(self.L.bb_debug_collide(self.h, stage))

    def debug_wait_limit(self, polls: int, abandon_block: bool = False):
        """Bound of the persistent kernels' grid-barrier waits (0 = default); abandon_block makes
        the colour-sweep kernel's last block leave so the other blocks' waits run out."""
        _check(self.L.bb_debug_wait_limit(self.h, polls, 1 if abandon_block else 0))

    def set_auto_regrow(self, max_pairs_per_body: int):
        """Rerun steps that overflowed the pair capacity with more capacity (0 = off)."""
        _check(self.L.bb_world_set_auto_regrow(self.h, max_pairs_per_body))

    def save_state(self) -> np.ndarray:
        """Image of the world's state (uint8): poses, velocities, persistent contacts, lists..."""
        n = ctypes.c_uint64()
        _check(self.L.bb_world_save_state(self.h, None, 0, ctypes.byref(n)))
        buf = np.empty(n.value, np.uint8)
        _check(self.L.bb_world_save_state(self.h, _ptr(buf), buf.nbytes, ctypes.byref(n)))
        return buf

    def load_state(self, image: np.ndarray):
        """Restore an image from save_state into this world (same capacity, same bodies)."""
        buf = np.ascontiguousarray(image, np.uint8)
        _check(self.L.bb_world_load_state(self.h, _ptr(buf), buf.nbytes))

    def clear(self):
        """Remove every body and shape (device buffers kept); clears the device error bits."""
        self._shape_cache = {}
        _check(self.L.bb_world_clear(self.h))

    def debug_read(self, which: str):
        code = DBG[which]
        cnt = ctypes.c_uint64()
        _check(self.L.bb_debug_read(self.h, code, None, 0, ctypes.byref(cnt)))
        n = cnt.value
        if which in ("leaf_aabb", "node_aabb", "body_inertia"):
            buf = np.empty(n, np.float32)
        elif which == "lbvh_child":
            buf = np.empty(n, np.int32)
        elif which == "manifolds":
            buf = np.empty(n, MANIFOLD_DTYPE)
        elif which == "contacts":
            buf = np.empty(n, CONTACT_DTYPE)
        else:
            buf = np.empty(n, np.uint32)
        _check(self.L.bb_debug_read(self.h, code, _ptr(buf), buf.nbytes, ctypes.byref(cnt)))
        return buf.reshape(-1, 6) if which == "body_inertia" else buf

    # ---- profiling --------------------------------------------------------------------------
    def set_profiling(self, on: bool):
        _check(self.L.bb_set_profiling(self.h, 1 if on else 0))

    def stage_times(self) -> dict:
        ms = np.zeros(32, np.float32)
        ns = _U32()
        names = ctypes.create_string_buffer(1024)
        _check(self.L.bb_read_stage_times(self.h, _ptr(ms), 32, ctypes.byref(ns), names, 1024))
        nm = names.raw.split(b"\0")[: ns.value]
        return {k.decode(): float(v) for k, v in zip(nm, ms[: ns.value])}


def voxel_shape_info(solid, voxel_size: float) -> dict:
    """What a voxel shape derives from its grid (solid[z, y, x]), computed on the host:
    grid origin (minus the centre of mass), box min/max, solid and surface counts, mass and
    inverse inertia (xx yy zz xy xz yz) at density 1, and the packed surface list."""
    L = load_library()
    g = np.ascontiguousarray(np.asarray(solid) != 0, dtype=np.uint8)
    nz, ny, nx = g.shape
    info = VoxelInfo()
    _check(L.bb_voxel_shape_info(nx, ny, nz, float(voxel_size), g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(info),
                                 None, 0))
    surf = np.zeros(info.surface_count, np.uint32)
    _check(L.bb_voxel_shape_info(nx, ny, nz, float(voxel_size), g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(info),
                                 surf.ctypes.data_as(ctypes.c_void_p), len(surf)))
    return {"grid_origin": np.array(info.grid_origin[:], np.float32), "box_min": np.array(info.box_min[:], np.float32),
            "box_max": np.array(info.box_max[:], np.float32), "solid_count": int(info.solid_count),
            "surface_count": int(info.surface_count), "unit_mass": np.float32(info.unit_mass),
            "unit_inv_inertia": np.array(info.unit_inv_inertia[:], np.float32), "surface": surf}


def world_from_scene(scene: dict, params: SolverParams | None = None, pairs_per_body: int = 16, **kw) -> World:
    """World holding every body of a scene, with its Morton bounds applied."""
    w = World(int(scene["n"]), pairs_per_body=pairs_per_body)
    w.add_scene(scene)
    p = params if params is not None else default_params()
    if not isinstance(p, SolverParams):
        p = SolverParams.from_buffer_copy(bytes(p))
    if scene.get("bounds") is not None:
        p.world_min[:] = scene["bounds"][0]
        p.world_extent[:] = scene["bounds"][1]
    w.set_params(p, **kw)
    return w


def scene_request_arrays(scene: dict, inertia_mode: int = INERTIA_EXPLICIT):
    """(shapes, bodies) ctypes arrays of a scene for a server request: one shape per distinct
    (type, half extents), body.shape indexing the shape table."""
    if scene.get("voxel_shapes"):
        raise ValueError("scene_request_arrays: served worlds take box and sphere shapes only")
    table: dict = {}
    idx = []
    for t, h in zip(scene["shape"].tolist(), scene["half"].tolist()):
        key = (int(t), float(h[0]), float(h[1]), float(h[2]))
        if key not in table:
            table[key] = len(table)
        idx.append(table[key])
    shapes = (ShapeDesc * len(table))()
    for key, k in table.items():
        shapes[k].type = key[0]
        shapes[k].half[:] = key[1:]
    n = int(scene["n"])
    bodies = (BodyDesc * n)()
    a = np.frombuffer(bodies, dtype=BODY_DTYPE, count=n)
    a["position"] = scene["pos"]
    a["rotation"] = scene["quat"]
    a["velocity"] = scene["vel"]
    a["omega"] = scene["omega"]
    a["shape"] = idx
    a["flags"] = scene["flags"]
    a["mass"] = scene["mass"]
    a["friction"] = scene["friction"]
    a["restitution"] = scene["restitution"]
    a["inertia_mode"] = inertia_mode
    a["inv_inertia"] = scene["inv_inertia"]
    return shapes, bodies


class Server:
    """Serving loop (bb_server_*): step requests for device-resident worlds, admitted by an HBM
    budget, overlapping on the device."""

    def __init__(self, hbm_budget_bytes: int, max_active: int = 64, pairs_per_body: int = 8, device: int = -1):
        self.L = load_library()
        d = ServerDesc(hbm_budget_bytes, max_active, pairs_per_body, device)
        h = ctypes.c_void_p()
        _check(self.L.bb_server_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def close(self):
        if self.h:
            _check(self.L.bb_server_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, world: int, steps: int, params: SolverParams, dt: float = 1.0 / 60.0, substeps: int = 1,
               scene: dict | None = None, arrays=None) -> int:
        """Queue `steps` steps of world `world`; a new world needs `scene` (or prebuilt `arrays`
        from scene_request_arrays, plus scene for its bounds)."""
        r = Request()
        r.world = world
        r.params = params if isinstance(params, SolverParams) else SolverParams.from_buffer_copy(bytes(params))
        r.dt = dt
        r.substeps = substeps
        r.steps = steps
        if scene is not None:
            shapes, bodies = arrays if arrays is not None else scene_request_arrays(scene)
            r.shapes = ctypes.cast(shapes, ctypes.POINTER(ShapeDesc))
            r.n_shapes = len(shapes)
            r.bodies = ctypes.cast(bodies, ctypes.POINTER(BodyDesc))
            r.n_bodies = len(bodies)
            b = scene.get("bounds") or ([-64.0] * 3, [128.0] * 3)
            r.world_min[:] = [float(v) for v in b[0]]
            r.world_extent[:] = [float(v) for v in b[1]]
        t = ctypes.c_uint64()
        _check(self.L.bb_server_submit(self.h, ctypes.byref(r), ctypes.byref(t)))
        return t.value

    def poll(self, ticket: int) -> dict:
        st = RequestStatus()
        _check(self.L.bb_server_poll(self.h, ticket, ctypes.byref(st)))
        return dict(done=bool(st.done), result=st.result, submit_s=st.submit_s, start_s=st.start_s,
                    finish_s=st.finish_s, error_flags=st.error_flags, error_site=st.error_site)

    def wait(self, ticket: int) -> dict:
        st = RequestStatus()
        _check(self.L.bb_server_wait(self.h, ticket, ctypes.byref(st)))
        return dict(done=bool(st.done), result=st.result, submit_s=st.submit_s, start_s=st.start_s,
                    finish_s=st.finish_s, error_flags=st.error_flags, error_site=st.error_site)

    def read_state(self, world: int, n: int) -> dict:
        out = dict(pos=np.empty((n, 3), np.float32), quat=np.empty((n, 4), np.float32),
                   vel=np.empty((n, 3), np.float32), omega=np.empty((n, 3), np.float32))
        cnt = _U32()
        _check(self.L.bb_server_read_state(self.h, world, _ptr(out["pos"]), _ptr(out["quat"]), _ptr(out["vel"]),
                                           _ptr(out["omega"]), ctypes.byref(cnt)))
        return out

    def stats(self) -> dict:
        st = ServerStats()
        _check(self.L.bb_server_get_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}


class RigidBodyManager:
    """Drop-in for the reference's beatbox::RigidBodyManager (src/rigid_body_manager.hpp:12-70).

    simulate() advances one fixed step (TIME_STEP = 0.01667 s, include/defines.hpp:354) in
    ``substeps`` pipeline passes; read_back_sim_config() returns the SimConfig-style counters.
    """

    TIME_STEP = 0.01667

    def __init__(self, max_bodies: int = 1024, pairs_per_body: int = 16):
        self.world = World(max_bodies, pairs_per_body=pairs_per_body)
        self._sim_config: dict = {}
        self.substeps = 1

    def create(self, name: str = "", iterations: int = 5) -> bool:
        self.world.set_params(iterations=iterations, relax_iterations=iterations)
        return True

    def simulate(self) -> bool:
        self.world.step(self.TIME_STEP, self.substeps)
        return True

    def read_back_sim_config(self) -> bool:
        self._sim_config = self.world.stats()
        return True

    def get_sim_config_reference(self) -> dict:
        return self._sim_config

    def skip_warm_starting_once(self):
        self.world.skip_warm_starting_once()

    def get_sim_flags(self) -> int:
        return int(self.world.params.flags)

    def set_sim_flags(self, flags: int) -> int:
        p = self.world.params
        p.flags |= flags
        self.world.set_params(p)
        return int(p.flags)

    def clear_sim_flags(self, flags: int) -> int:
        p = self.world.params
        p.flags &= ~flags
        self.world.set_params(p)
        return int(p.flags)

    def set_sim_type(self, solver: int):
        self.world.set_params(solver=solver)

    def get_sim_type(self) -> int:
        return int(self.world.params.solver)
