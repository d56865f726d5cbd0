"""Seeded synthetic scenes for the rigid-body pipeline.

The reference builds its scenes in C++ (src/scene_manager.hpp:114-823) with an unseeded
std::mt19937 (scene_manager.hpp:832-833), so they are not reproducible.  These generators use a
counter-based splitmix64 stream instead: the same seed gives the same bodies on every machine.
They stand in for the workloads the benchmark is quoted on (no public dataset exists for them):

* ``box_grid``     -- 1,000 unit boxes in a jittered 10x10x10 grid over a ground box.
* ``mixed_column`` -- 100k boxes and spheres in a 60x60x200 m column inside a 5-wall container.
* ``pyramids``     -- 1,000 box pyramids of 1,000 boxes each on a 32x32 grid.
* ``batch_worlds`` -- many independent small piles (world id per body).
* ``voxel_pile``   -- concave voxel bodies (L, cross, hollow frame) dropped on a ground box, the
                      kind of scene the reference's voxel showcase builds (scene_manager.hpp:574-).

A scene is a dict of numpy arrays, one row per body, ready for ``World.add_bodies`` and for the
oracle.  Static bodies have mass 0, inverse mass 0 and zero inverse inertia.
"""
from __future__ import annotations

import math

import numpy as np

BODY_DYNAMIC = 1 << 1
BODY_GRAVITY = 1 << 2
SHAPE_BOX = 0
SHAPE_SPHERE = 1
SHAPE_VOXEL = 2

_M64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    """n uniform doubles in [lo, hi) from counter (seed, stream, i)."""
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x632BE59BD9B4E019 + stream * 0x9E3779B97F4A7C15) & _M64)
        ctr = np.arange(n, dtype=np.uint64) + base
        u = (splitmix64(ctr) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    return lo + (hi - lo) * u


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    """n standard normal doubles (Box-Muller on two uniform streams)."""
    u1 = np.maximum(uniform(seed, stream, n), 1e-300)
    u2 = uniform(seed, stream + 1_000_003, n)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def random_rotations(seed: int, stream: int, n: int) -> np.ndarray:
    """Uniform rotations on SO(3) (Shoemake), quaternion x, y, z, w."""
    u1 = uniform(seed, stream, n)
    u2 = uniform(seed, stream + 1, n) * 2 * math.pi
    u3 = uniform(seed, stream + 2, n) * 2 * math.pi
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    return np.stack([a * np.sin(u2), a * np.cos(u2), b * np.sin(u3), b * np.cos(u3)], axis=1)


def yaw_rotations(angles: np.ndarray) -> np.ndarray:
    h = 0.5 * angles
    z = np.zeros_like(h)
    return np.stack([z, np.sin(h), z, np.cos(h)], axis=1)


def box_inverse_inertia(mass: np.ndarray, half: np.ndarray, mode: str) -> np.ndarray:
    """Body-frame inverse inertia diagonal of solid boxes.

    mode "physical": I_xx = m (h^2 + d^2) / 12 with full sizes.
    mode "reference": cuboid_get_inverse_intertia(inv_mass, min, max) as the reference scene
    builder calls it (src/scene_manager.hpp:861, include/math.hpp:106-130), in float32.
    """
    size = (2.0 * half).astype(np.float32)
    w, h, d = size[:, 0], size[:, 1], size[:, 2]
    out = np.zeros_like(size)
    dyn = mass > 0
    if mode == "physical":
        m = mass.astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            out[:, 0] = np.where(dyn, 12.0 / (m * (h * h + d * d)), 0)
            out[:, 1] = np.where(dyn, 12.0 / (m * (w * w + d * d)), 0)
            out[:, 2] = np.where(dyn, 12.0 / (m * (w * w + h * h)), 0)
        return out.astype(np.float32)
    if mode == "reference":
        inv_m = np.where(dyn, np.float32(1.0) / np.where(dyn, mass, 1).astype(np.float32), 0).astype(np.float32)
        twelfth = np.float32(1.0) / np.float32(12.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            ixx = twelfth * inv_m * (h * h + d * d)
            iyy = twelfth * inv_m * (w * w + d * d)
            izz = twelfth * inv_m * (w * w + h * h)
            out[:, 0] = np.where(dyn, np.float32(1.0) / ixx, 0)
            out[:, 1] = np.where(dyn, np.float32(1.0) / iyy, 0)
            out[:, 2] = np.where(dyn, np.float32(1.0) / izz, 0)
        return out.astype(np.float32)
    raise ValueError(mode)


def sphere_inverse_inertia(mass: np.ndarray, radius: np.ndarray, mode: str) -> np.ndarray:
    dyn = mass > 0
    if mode == "reference":
        return box_inverse_inertia(mass, np.repeat(radius[:, None], 3, axis=1), "reference")
    with np.errstate(divide="ignore", invalid="ignore"):
        v = np.where(dyn, 5.0 / (2.0 * mass.astype(np.float64) * radius.astype(np.float64) ** 2), 0)
    return np.repeat(v[:, None], 3, axis=1).astype(np.float32)


class SceneBuilder:
    """Accumulates bodies as arrays."""

    def __init__(self, inertia: str = "physical"):
        self.inertia = inertia
        self.parts: list[dict] = []
        self.voxel_shapes: list[dict] = []  # {"solid": uint8[z, y, x], "voxel_size": float, "info": ...}
        self.bounds = None  # optional (world_min[3], world_extent[3]) for Morton codes

    def add(self, pos, quat, half, shape, flags, mass, friction=0.5, restitution=0.0, vel=None, omega=None):
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        n = pos.shape[0]
        quat = np.asarray(quat, np.float64).reshape(n, 4)
        half = np.asarray(half, np.float64).reshape(n, 3)
        shape = np.broadcast_to(np.asarray(shape, np.uint32), (n,)).copy()
        flags = np.broadcast_to(np.asarray(flags, np.uint32), (n,)).copy()
        mass = np.broadcast_to(np.asarray(mass, np.float64), (n,)).copy()
        dyn = (flags & BODY_DYNAMIC) != 0
        mass = np.where(dyn, mass, 0.0)
        inv_mass = np.where(dyn & (mass > 0), 1.0 / np.where(mass > 0, mass, 1.0), 0.0)
        m32 = mass.astype(np.float32)
        ii = np.zeros((n, 3), np.float32)
        box = shape == SHAPE_BOX
        if box.any():
            ii[box] = box_inverse_inertia(m32[box], half[box].astype(np.float32), self.inertia)
        sph = ~box
        if sph.any():
            ii[sph] = sphere_inverse_inertia(m32[sph], half[sph, 0].astype(np.float32), self.inertia)
        ii[~dyn] = 0
        if self.inertia == "reference":
            inv_mass = np.where(dyn, (np.float32(1.0) / np.where(dyn, m32, 1).astype(np.float32)), 0)
        self.parts.append(dict(
            pos=pos.astype(np.float32), quat=quat.astype(np.float32), half=half.astype(np.float32),
            shape=shape, flags=flags, mass=m32, inv_mass=np.asarray(inv_mass, np.float32), inv_inertia=ii,
            inv_inertia_off=np.zeros((n, 3), np.float32), voxel=np.zeros(n, np.uint32),
            friction=np.broadcast_to(np.asarray(friction, np.float32), (n,)).copy(),
            restitution=np.broadcast_to(np.asarray(restitution, np.float32), (n,)).copy(),
            vel=np.zeros((n, 3), np.float32) if vel is None else np.asarray(vel, np.float32).reshape(n, 3),
            omega=np.zeros((n, 3), np.float32) if omega is None else np.asarray(omega, np.float32).reshape(n, 3),
        ))

    def add_voxel_shape(self, solid, voxel_size: float) -> int:
        """Register an occupancy grid solid[z, y, x]; returns its index for add_voxel."""
        from . import voxel_shape_info  # the library's host build (centre of mass, inertia)
        g = np.ascontiguousarray(np.asarray(solid) != 0, dtype=np.uint8)
        self.voxel_shapes.append({"solid": g, "voxel_size": float(voxel_size), "info": voxel_shape_info(g, voxel_size)})
        return len(self.voxel_shapes) - 1

    def add_voxel(self, pos, quat, shape_index, flags, density=1000.0, friction=0.5, vel=None, omega=None):
        """Voxel bodies of one registered shape.  Mass = density * unit mass; the inverse inertia
        (diagonal and off-diagonal) is the shape's unit one scaled by unit_mass / mass in float32,
        the same arithmetic the library applies to a voxel body added without explicit inertia."""
        info = self.voxel_shapes[shape_index]["info"]
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        n = pos.shape[0]
        flags = np.broadcast_to(np.asarray(flags, np.uint32), (n,)).copy()
        dyn = (flags & BODY_DYNAMIC) != 0
        mass = np.where(dyn, np.float32(density) * info["unit_mass"], np.float32(0)).astype(np.float32)
        scale = np.where(dyn, info["unit_mass"] / np.where(dyn, mass, np.float32(1)), np.float32(0)).astype(np.float32)
        ui = info["unit_inv_inertia"]
        ii = (ui[None, :3] * scale[:, None]).astype(np.float32)
        io = (ui[None, 3:] * scale[:, None]).astype(np.float32)
        half = 0.5 * (info["box_max"] - info["box_min"])
        self.parts.append(dict(
            pos=pos.astype(np.float32), quat=np.asarray(quat, np.float64).reshape(n, 4).astype(np.float32),
            half=np.tile(half.astype(np.float32), (n, 1)), shape=np.full(n, SHAPE_VOXEL, np.uint32), flags=flags,
            mass=mass, inv_mass=np.where(dyn, np.float32(1) / np.where(dyn, mass, np.float32(1)), 0).astype(np.float32),
            inv_inertia=ii, inv_inertia_off=io, voxel=np.full(n, shape_index, np.uint32),
            friction=np.broadcast_to(np.asarray(friction, np.float32), (n,)).copy(),
            restitution=np.zeros(n, np.float32),
            vel=np.zeros((n, 3), np.float32) if vel is None else np.asarray(vel, np.float32).reshape(n, 3),
            omega=np.zeros((n, 3), np.float32) if omega is None else np.asarray(omega, np.float32).reshape(n, 3),
        ))

    def add_static_box(self, center, half, friction=0.5):
        self.add([center], [[0, 0, 0, 1]], [half], SHAPE_BOX, 0, 0.0, friction=friction)

    def build(self) -> dict:
        keys = self.parts[0].keys()
        scene = {k: np.ascontiguousarray(np.concatenate([p[k] for p in self.parts])) for k in keys}
        scene["n"] = scene["pos"].shape[0]
        scene["bounds"] = self.bounds
        if self.voxel_shapes:
            scene["voxel_shapes"] = [{"solid": v["solid"], "voxel_size": v["voxel_size"]} for v in self.voxel_shapes]
        return scene


def box_grid(n_side: int = 10, seed: int = 0, density: float = 1000.0, half: float = 0.5, spacing: float = 1.1,
             jitter: float = 0.05, friction: float = 0.5, inertia: str = "physical", layers: int | None = None) -> dict:
    """Jittered grid of boxes dropped on a ground box (1,000 boxes at the defaults).

    Layer j sits at y = half + 0.1 + spacing * j (0.1 m clearance above the ground top y = 0);
    x/z centred on 0; per-axis jitter U(+-jitter); yaw U[0, 2 pi).  Ground: static box centred
    at (0, -50, 0) with half extent 50 (the reference floor, src/scene_manager.hpp:171).
    """
    layers = n_side if layers is None else layers
    ix, iy, iz = np.meshgrid(np.arange(n_side), np.arange(layers), np.arange(n_side), indexing="xy")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    order = np.lexsort((ix, iz, iy))
    ix, iy, iz = ix[order], iy[order], iz[order]
    n = ix.size
    off = (n_side - 1) * spacing * 0.5
    pos = np.stack([ix * spacing - off, half + 0.1 + iy * spacing, iz * spacing - off], axis=1).astype(np.float64)
    pos += np.stack([uniform(seed, 1 + k, n, -jitter, jitter) for k in range(3)], axis=1)
    quat = yaw_rotations(uniform(seed, 4, n, 0.0, 2 * math.pi))
    sb = SceneBuilder(inertia)
    sb.add_static_box([0.0, -50.0, 0.0], [50.0, 50.0, 50.0], friction=friction)
    mass = density * (2 * half) ** 3
    sb.add(pos, quat, np.full((n, 3), half), SHAPE_BOX, BODY_DYNAMIC | BODY_GRAVITY, mass, friction=friction)
    return sb.build()


def mixed_column(n_bodies: int = 100_000, seed: int = 0, density: float = 1000.0, friction: float = 0.5,
                 inertia: str = "physical", box_fraction: float = 0.6) -> dict:
    """Boxes (half extents U[0.2, 0.8] per axis) and spheres (radius lognormal mu=ln 0.4,
    sigma=0.3, clipped to [0.1, 0.9]) on a jittered lattice filling a 60x60x200 m column
    (x, z in [-30, 30], y in [1, 201]) with uniform random orientations, inside a static
    container: floor (top at y=0) and four walls 0.5 m thick, 25 m high, around 61x61 m."""
    n_box = int(round(n_bodies * box_fraction))
    n_sph = n_bodies - n_box
    side = 30
    per_layer = side * side
    layers = (n_bodies + per_layer - 1) // per_layer
    pitch_xz = 60.0 / side
    pitch_y = 200.0 / layers
    k = np.arange(n_bodies)
    ly, rem = np.divmod(k, per_layer)
    lz, lx = np.divmod(rem, side)
    pos = np.stack([-30.0 + (lx + 0.5) * pitch_xz, 1.0 + (ly + 0.5) * pitch_y, -30.0 + (lz + 0.5) * pitch_xz], axis=1)
    pos += np.stack([uniform(seed, 10 + a, n_bodies, -0.1, 0.1) for a in range(3)], axis=1)
    perm = np.argsort(uniform(seed, 20, n_bodies), kind="stable")  # shuffle box/sphere slots
    pos = pos[perm]
    quat = random_rotations(seed, 30, n_bodies)
    half_box = np.stack([uniform(seed, 40 + a, n_box, 0.2, 0.8) for a in range(3)], axis=1)
    radius = np.clip(np.exp(math.log(0.4) + 0.3 * normal(seed, 50, n_sph)), 0.1, 0.9)
    sb = SceneBuilder(inertia)
    sb.add_static_box([0.0, -0.5, 0.0], [31.0, 0.5, 31.0], friction=friction)
    for sx in (-1, 1):
        sb.add_static_box([sx * 30.75, 12.5, 0.0], [0.25, 12.5, 31.0], friction=friction)
        sb.add_static_box([0.0, 12.5, sx * 30.75], [31.0, 12.5, 0.25], friction=friction)
    flags = BODY_DYNAMIC | BODY_GRAVITY
    sb.add(pos[:n_box], quat[:n_box], half_box, SHAPE_BOX, flags,
           density * 8.0 * half_box.prod(axis=1), friction=friction)
    sb.add(pos[n_box:], quat[n_box:], np.repeat(radius[:, None], 3, axis=1), SHAPE_SPHERE, flags,
           density * (4.0 / 3.0) * math.pi * radius ** 3, friction=friction)
    sb.bounds = ([-32.0, -2.0, -32.0], [64.0, 206.0, 64.0])
    return sb.build()


def pyramids(n_pyramids: int = 1000, boxes_per: int = 1000, seed: int = 0, density: float = 1000.0,
             friction: float = 0.5, inertia: str = "physical", cell: float = 20.0, grid: int = 32,
             base: int = 18, gap: float = 0.001) -> dict:
    """Box pyramids (base 18x18 tapering, first ``boxes_per`` boxes in layer/row-major order)
    on a grid x grid layout of cells ``cell`` m apart (first n_pyramids cells, row-major), unit
    boxes with a 1 mm gap, initial velocity N(0, 0.01) m/s per component, over a ground box."""
    offs = []
    layer = 0
    while len(offs) < boxes_per:
        s = base - layer
        if s <= 0:
            break
        for r in range(s):
            for c in range(s):
                if len(offs) < boxes_per:
                    offs.append(((c - (s - 1) / 2) * (1 + gap), 0.5 + gap / 2 + layer * (1 + gap),
                                 (r - (s - 1) / 2) * (1 + gap)))
        layer += 1
    offs = np.asarray(offs)
    cells = np.arange(n_pyramids)
    cz, cx = np.divmod(cells, grid)
    extent = grid * cell
    centers = np.stack([cx * cell - extent / 2 + cell / 2, np.zeros(n_pyramids), cz * cell - extent / 2 + cell / 2], 1)
    pos = (centers[:, None, :] + offs[None, :, :]).reshape(-1, 3)
    n = pos.shape[0]
    vel = np.stack([0.01 * normal(seed, 60 + 2 * a, n) for a in range(3)], axis=1)
    sb = SceneBuilder(inertia)
    sb.add_static_box([0.0, -0.5, 0.0], [extent / 2 + 10, 0.5, extent / 2 + 10], friction=friction)
    sb.add(pos, np.tile([0, 0, 0, 1.0], (n, 1)), np.full((n, 3), 0.5), SHAPE_BOX, BODY_DYNAMIC | BODY_GRAVITY,
           density, friction=friction, vel=vel)
    sb.bounds = ([-extent / 2 - 12, -2.0, -extent / 2 - 12], [extent + 24, extent + 24, extent + 24])
    return sb.build()


def pile(n_bodies: int, seed: int = 0, sphere_fraction: float = 0.4, density: float = 1000.0,
         friction: float = 0.5, inertia: str = "physical") -> dict:
    """A config-1 style pile scaled to n_bodies: unit boxes (half extent 0.5) and spheres
    (radius 0.5) in a jittered grid, side = ceil(n^(1/3)) columns per axis and as many layers as
    needed, 1.1 m spacing, 0.1 m above the ground top, per-axis jitter U(+-0.05), yaw U[0, 2 pi);
    a random sphere_fraction of the slots holds spheres.  Ground: static box centred at
    (0, -50, 0), half extent 50.  The scene's Morton box covers the pile with a 4 m margin."""
    side = max(1, int(math.ceil(n_bodies ** (1.0 / 3.0) - 1e-9)))
    per_layer = side * side
    k = np.arange(n_bodies)
    ly, rem = np.divmod(k, per_layer)
    lz, lx = np.divmod(rem, side)
    off = (side - 1) * 1.1 * 0.5
    pos = np.stack([lx * 1.1 - off, 0.6 + ly * 1.1, lz * 1.1 - off], axis=1).astype(np.float64)
    pos += np.stack([uniform(seed, 1 + a, n_bodies, -0.05, 0.05) for a in range(3)], axis=1)
    quat = yaw_rotations(uniform(seed, 4, n_bodies, 0.0, 2 * math.pi))
    is_sph = uniform(seed, 5, n_bodies) < sphere_fraction
    flags = BODY_DYNAMIC | BODY_GRAVITY
    sb = SceneBuilder(inertia)
    sb.add_static_box([0.0, -50.0, 0.0], [50.0, 50.0, 50.0], friction=friction)
    box = ~is_sph
    if box.any():
        sb.add(pos[box], quat[box], np.full((int(box.sum()), 3), 0.5), SHAPE_BOX, flags, density * 1.0,
               friction=friction)
    if is_sph.any():
        ns = int(is_sph.sum())
        sb.add(pos[is_sph], quat[is_sph], np.full((ns, 3), 0.5), SHAPE_SPHERE, flags,
               density * (4.0 / 3.0) * math.pi * 0.125, friction=friction)
    height = 0.6 + (int(ly.max()) + 1) * 1.1
    sb.bounds = ([-off - 4.0, -4.0, -off - 4.0], [2 * off + 8.0, height + 8.0, 2 * off + 8.0])
    return sb.build()


def batch_sizes(n_worlds: int, seed: int = 0, lo: int = 16, hi: int = 2048) -> np.ndarray:
    """Body counts of a batch: floor(exp(U(ln lo, ln hi))) per world."""
    u = uniform(seed, 90, n_worlds, math.log(lo), math.log(hi))
    return np.floor(np.exp(u)).astype(np.int64)


# ---- voxel (concave) bodies --------------------------------------------------------------
def voxel_l_shape(n: int = 4, thick: int = 2) -> np.ndarray:
    """An L: an n x n x thick slab with the (n-1) x (n-1) upper-right block removed, grid [z, y, x]."""
    g = np.zeros((thick, n, n), np.uint8)
    g[:, 0, :] = 1
    g[:, :, 0] = 1
    return g


def voxel_cross(n: int = 5, thick: int = 1) -> np.ndarray:
    """A plus sign of arm width 1 in an n x n plane, thick cells deep, grid [z, y, x]."""
    g = np.zeros((thick, n, n), np.uint8)
    g[:, n // 2, :] = 1
    g[:, :, n // 2] = 1
    return g


def voxel_frame(n: int = 5, thick: int = 1) -> np.ndarray:
    """A hollow square frame (border one cell wide) in an n x n plane, grid [z, y, x]."""
    g = np.ones((thick, n, n), np.uint8)
    g[:, 1:-1, 1:-1] = 0
    return g


def voxel_pile(n_bodies: int = 60, seed: int = 0, voxel_size: float = 0.2, density: float = 1000.0,
               friction: float = 0.5, spacing: float = 1.6, height: float = 1.2, layer: float = 1.5) -> dict:
    """Concave voxel bodies (L, cross, hollow frame, cycling) with uniform random orientations,
    jittered on a grid (spacing and layer apart, so no two overlap at the start) over a static
    ground box (top at y = 0)."""
    sb = SceneBuilder()
    per = max(1, int(math.ceil(math.sqrt(n_bodies / 3.0))))
    ground = max(50.0, 0.5 * spacing * per + 10.0)
    sb.add_static_box([0, -ground, 0], [ground, ground, ground], friction=friction)
    shapes = [sb.add_voxel_shape(g, voxel_size) for g in (voxel_l_shape(), voxel_cross(), voxel_frame())]
    k = np.arange(n_bodies)
    lay, rem = k // (per * per), k % (per * per)
    gx, gz = rem % per, rem // per
    half = 0.5 * spacing * (per - 1)
    pos = np.stack([-half + gx * spacing + uniform(seed, 1, n_bodies, -0.05, 0.05),
                    height + lay * layer + uniform(seed, 2, n_bodies, 0.0, 0.1),
                    -half + gz * spacing + uniform(seed, 3, n_bodies, -0.05, 0.05)], axis=1)
    quat = random_rotations(seed, 10, n_bodies)
    for si in range(len(shapes)):
        sel = k % len(shapes) == si
        if sel.any():
            sb.add_voxel(pos[sel], quat[sel], shapes[si], BODY_DYNAMIC | BODY_GRAVITY, density, friction)
    top = height + (int(lay.max()) + 2) * layer if n_bodies else height
    span = 0.5 * spacing * per + 4.0
    sb.bounds = ([-span, -2.0, -span], [2 * span, top + 4.0, 2 * span])
    return sb.build()
