"""The reference's demo scenes 1..7 as scene dicts (src/scene_manager.hpp:114-823).

Each scene is built the way the reference's SceneManager::load_scene turns its body list into a
world (src/scene_manager.hpp:850-887): inverse mass 1 / mass, box inverse inertia from
cuboid_get_inverse_intertia(inv_mass, min, max) (the builder's quirk, ``inertia="reference"``),
voxel bodies' mass and inertia from their voxel sum.  Materials, lights and the emissive panel's
colour are render state and are not kept; the panels stay as the static boxes they are.

Deliberate differences, each because the reference's input is not reproducible or not a
rotation:
  * scene_2 draws its 1,000 cube positions from an unseeded std::mt19937
    (scene_manager.hpp:832-833); here they come from the seeded splitmix64 stream;
  * scene_1 passes four unnormalised quaternions (e.g. (0, 1, 1, 0.8)); the reference uses
    them as given until its first integration renormalises them.  They are normalised here.

``reference_scene(k)`` builds scene k; ``beatbox.io.load_reference_scene(k)`` reads the same
scene from the data files shipped in ``beatbox/scene_data`` (written by make_scene_data.py).
"""
from __future__ import annotations

import math

import numpy as np

from .scenes import BODY_DYNAMIC, BODY_GRAVITY, SHAPE_BOX, SceneBuilder, uniform

DYN = BODY_DYNAMIC | BODY_GRAVITY


def _q(x, y, z, w):
    q = np.array([x, y, z, w], np.float64)
    return (q / np.linalg.norm(q)).tolist()


def _static(sb, pos, half, friction, restitution=0.0, quat=(0, 0, 0, 1)):
    sb.add([pos], [quat], [half], SHAPE_BOX, 0, 0.0, friction=friction, restitution=restitution)


def _cube(sb, pos, quat, half, mass, friction, restitution, omega=None):
    sb.add([pos], [quat], [half], SHAPE_BOX, DYN, mass, friction=friction, restitution=restitution,
           omega=None if omega is None else [omega])


def _ground(sb, friction, restitution=0.0):
    _static(sb, (0.0, -50.0, 0.0), (50.0, 50.0, 50.0), friction, restitution)


def scene_1() -> dict:
    """Ground and 18 cubes of assorted sizes, orientations, restitution and friction
    (scene_manager.hpp:114-191)."""
    sb = SceneBuilder("reference")
    _ground(sb, 0.5, 0.5)
    h = (0.5, 0.5, 0.5)
    rows = [  # position, quaternion (x, y, z, w), half extents, mass, restitution, friction, omega
        ((-0.5, 2.0, -0.5), (0.4572, 0.0, -0.4572, -0.7629), h, 5.0, 0.7, 0.3, None),
        ((-3.0, 5.0, -1.0), (0.0, 0.0, 0.0, 1.0), (1.0, 1.0, 1.0), 5.0, 0.1, 0.6, (0.0, 0.0, 10.0)),
        ((0.3, 1.7, 0.3), (-0.4572, 0.0, 0.4572, -0.7629), h, 2.0, 0.3, 0.6, None),
        ((-0.5, 0.25, 0.5), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.4, 0.2, None),
        ((2.5, 3.0, 2.5), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.5, 0.5, None),
        ((1.5, 3.0, 2.3), (0.0, 0.0, 0.5, 1.0), h, 5.0, 0.6, 0.7, None),
        ((-2.5, 3.0, 2.5), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.7, 0.8, None),
        ((-2.5, 3.25, 1.5), (0.5, 0.0, 0.0, 1.0), h, 5.0, 0.8, 0.9, None),
        ((3.5, 2.0, 0.5), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.9, 0.6, None),
        ((2.5, 2.0, -0.2), (0.0, 1.0, 1.0, 0.8), h, 5.0, 0.9, 0.5, None),
        ((4.0, 2.5, -2.0), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.8, 0.5, None),
        ((5.0, 2.5, -2.7), (0.0, 1.0, 1.0, 0.8), h, 5.0, 0.7, 0.4, None),
        ((6.0, 3.5, 0.0), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.6, 0.7, None),
        ((5.0, 3.5, 0.7), (0.0, 1.0, 1.0, 0.8), h, 5.0, 0.5, 0.3, None),
        ((6.5, 1.5, 0.0), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.4, 0.6, None),
        ((7.5, 1.5, 0.9), (0.0, 1.0, 1.0, 0.8), h, 5.0, 0.3, 0.9, None),
        ((6.9, 2.5, 4.5), (0.0, 0.0, 0.0, 1.0), h, 5.0, 0.2, 0.3, None),
        ((5.8, 3.5, 4.5), (0.0, 1.0, 0.0, -0.5), h, 5.0, 0.1, 0.3, None),
    ]
    for pos, q, half, m, e, mu, om in rows:
        _cube(sb, pos, _q(*q), half, m, mu, e, om)
    return sb.build()


def scene_2(seed: int = 0, n_body: int = 1000) -> dict:
    """Ground and 1,000 cubes at uniform random positions x, z in [-15, 15], y in [2, 7]
    (scene_manager.hpp:193-268; seeded here)."""
    sb = SceneBuilder("reference")
    _ground(sb, 0.5, 0.5)
    pos = np.stack([uniform(seed, 1, n_body, -15.0, 15.0), uniform(seed, 2, n_body, 2.0, 7.0),
                    uniform(seed, 3, n_body, -15.0, 15.0)], axis=1)
    sb.add(pos, np.tile([0, 0, 0, 1.0], (n_body, 1)), np.full((n_body, 3), 0.5), SHAPE_BOX, DYN, 5.0,
           friction=0.5, restitution=0.5)
    return sb.build()


def scene_3() -> dict:
    """Three cube towers of 5, 8 and 12 (1 mm settle gap per level) and the static panel
    (scene_manager.hpp:270-353): tall stacks must stay upright."""
    sb = SceneBuilder("reference")
    _ground(sb, 0.5)
    _static(sb, (0.0, 22.0, 14.0), (5.0, 0.2, 5.0), 0.5)
    for x, height in ((-6.0, 5), (0.0, 8), (6.0, 12)):
        for i in range(height):
            _cube(sb, (x, 0.5 + i * 1.001, 14.0), (0, 0, 0, 1), (0.5, 0.5, 0.5), 5.0, 0.5, 0.0)
    return sb.build()


def scene_4() -> dict:
    """Two static ramps (15 and 30 degrees, friction 1) with cube pairs of friction 0.04, 0.25
    and 1.0 and a 2-cube tower (scene_manager.hpp:355-470): a cube slides iff
    sqrt(mu_cube * 1) < tan(theta)."""
    sb = SceneBuilder("reference")
    _ground(sb, 1.0)
    _static(sb, (0.0, 20.0, 14.0), (5.0, 0.2, 5.0), 1.0)
    deg = 3.14159265 / 180.0
    th_a, th_b = 15.0 * deg, 30.0 * deg
    q_a = [0.0, 0.0, math.sin(th_a * 0.5), math.cos(th_a * 0.5)]
    q_b = [0.0, 0.0, -math.sin(th_b * 0.5), math.cos(th_b * 0.5)]
    xl_a, yl_a = (math.cos(th_a), math.sin(th_a)), (-math.sin(th_a), math.cos(th_a))
    xl_b, yl_b = (math.cos(th_b), -math.sin(th_b)), (math.sin(th_b), math.cos(th_b))
    ramp_a, ramp_b = (-7.0, 2.3, 14.0), (7.0, 3.9, 14.0)
    _static(sb, ramp_a, (7.0, 0.4, 4.5), 1.0, quat=q_a)
    _static(sb, ramp_b, (7.0, 0.4, 4.5), 1.0, quat=q_b)

    def cube(c, xl, yl, q, u, z, mu, lift):
        _cube(sb, (c[0] + u * xl[0] + lift * yl[0], c[1] + u * xl[1] + lift * yl[1], z), q, (0.5, 0.5, 0.5), 5.0,
              mu, 0.0)

    lift0 = 0.4 + 0.5 + 0.005
    for u, z, mu in ((3.5, 16.2, 0.04), (3.5, 17.8, 0.04), (1.75, 13.4, 0.25), (1.75, 15.0, 0.25), (0.0, 10.6, 1.0),
                     (0.0, 12.2, 1.0)):
        cube(ramp_a, xl_a, yl_a, q_a, u, z, mu, lift0)
    cube(ramp_a, xl_a, yl_a, q_a, 0.0, 10.6, 1.0, lift0 + 1.005)
    for u, z, mu in ((-3.5, 16.2, 0.04), (-3.5, 17.8, 0.04), (-1.75, 13.4, 0.25), (-1.75, 15.0, 0.25),
                     (0.0, 10.6, 1.0), (0.0, 12.2, 1.0)):
        cube(ramp_b, xl_b, yl_b, q_b, u, z, mu, lift0)
    return sb.build()


def _grid(dims, pred) -> np.ndarray:
    """Occupancy grid [z, y, x] of dims (x, y, z) from pred(x, y, z)."""
    nx, ny, nz = dims
    g = np.zeros((nz, ny, nx), np.uint8)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                g[z, y, x] = 1 if pred(x, y, z) else 0
    return g


def _voxel_shapes(sb, with_frame: bool):
    vs = 0.5
    shapes = {
        "l": sb.add_voxel_shape(_grid((6, 6, 2), lambda x, y, z: y < 2 or x < 2), vs),
        "cross": sb.add_voxel_shape(_grid((6, 6, 2), lambda x, y, z: 2 <= x < 4 or 2 <= y < 4), vs),
    }
    if with_frame:
        shapes["frame"] = sb.add_voxel_shape(_grid((8, 8, 2), lambda x, y, z: not (2 <= x < 6 and 2 <= y < 6)), vs)
    return shapes


Q_ID = (0.0, 0.0, 0.0, 1.0)
Q_X90 = (0.7071, 0.0, 0.0, 0.7071)


def scene_5() -> dict:
    """Concave voxel bodies (L, cross, hollow frame; 0.5 m voxels, density 2) piled beside a
    static post, and a frame that threads onto the post (scene_manager.hpp:578-660)."""
    sb = SceneBuilder("reference")
    _ground(sb, 0.6)
    _static(sb, (0.0, 22.0, 14.0), (5.0, 0.2, 5.0), 0.6)
    _static(sb, (8.0, 4.0, 14.0), (0.35, 4.0, 0.35), 0.6)
    s = _voxel_shapes(sb, True)
    for name, pos, q in (("l", (-6.0, 2.5, 13.0), Q_ID), ("l", (-5.4, 5.5, 14.6), Q_X90), ("l", (-2.0, 8.0, 13.8), Q_ID),
                         ("cross", (-3.5, 2.5, 14.8), Q_ID), ("cross", (-4.5, 11.0, 14.0), Q_X90),
                         ("cross", (0.5, 4.0, 14.2), Q_ID), ("frame", (-1.0, 12.5, 14.4), Q_ID),
                         ("frame", (2.5, 7.0, 13.4), Q_X90), ("frame", (8.0, 11.0, 14.0), Q_X90)):
        sb.add_voxel([pos], [_q(*q)], s[name], DYN, density=2.0, friction=0.6)
    return sb.build()


def scene_6() -> dict:
    """Deterministic voxel stability probes: an L flat on the floor, an L leaning on a static
    block, a tangle, a stack and a cantilevered stack (scene_manager.hpp:662-737)."""
    sb = SceneBuilder("reference")
    _ground(sb, 0.6)
    _static(sb, (0.0, 22.0, 14.0), (5.0, 0.2, 5.0), 0.6)
    _static(sb, (0.8, 1.0, 14.0), (0.5, 1.0, 2.0), 0.6)
    s = _voxel_shapes(sb, False)
    q_lean = (0.0, 0.0, 0.2588, 0.9659)
    q_tilt = (0.2164, 0.0, 0.0, 0.9763)
    for name, pos, q in (("l", (-6.0, 0.51, 14.0), Q_X90), ("l", (-0.9, 1.65, 14.0), q_lean),
                         ("cross", (6.0, 0.51, 14.0), Q_X90), ("l", (6.2, 1.45, 14.3), q_tilt),
                         ("l", (7.3, 1.30, 13.8), q_lean), ("cross", (-12.0, 0.51, 14.0), Q_X90),
                         ("l", (-12.0, 1.56, 14.0), Q_X90), ("cross", (-18.0, 0.51, 14.0), Q_X90),
                         ("l", (-17.2, 1.56, 14.6), Q_X90)):
        sb.add_voxel([pos], [_q(*q)], s[name], DYN, density=2.0, friction=0.6)
    return sb.build()


def scene_7() -> dict:
    """Box pool (scene_manager.hpp:739-823): 432 unit cubes in 12 waves of 6 x 6 rain into an
    8 x 8 m pit with 10 m walls, with index-hashed jitter and tilts.  The reference's success
    criterion: every cube asleep, no fresh contact, max speed 0."""
    sb = SceneBuilder("reference")
    _ground(sb, 0.6)
    _static(sb, (0.0, 50.0, 14.0), (8.0, 0.2, 8.0), 0.6)
    for pos, half in (((4.25, 5.0, 14.0), (0.25, 5.0, 4.5)), ((-4.25, 5.0, 14.0), (0.25, 5.0, 4.5)),
                      ((0.0, 5.0, 18.25), (4.5, 5.0, 0.25)), ((0.0, 5.0, 9.75), (4.5, 5.0, 0.25))):
        _static(sb, pos, half, 0.6)
    f32 = np.float32
    pos, quat = [], []
    for iy in range(12):
        for iz in range(6):
            for ix in range(6):
                h1 = ix * 3 + iy * 5 + iz * 7
                h2 = ix * 7 + iy * 3 + iz * 5
                h3 = ix * 5 + iy * 7 + iz * 3
                jx = (f32(h1 % 11) - f32(5.0)) * f32(0.05)
                jz = (f32(h2 % 11) - f32(5.0)) * f32(0.05)
                jy = (f32(h3 % 11) - f32(5.0)) * f32(0.20)
                phi = f32(h3 % 16) * f32(0.3927)
                ang = f32(0.07) + f32(h1 % 7) * f32(0.025)
                sh = np.sin(f32(0.5) * ang, dtype=f32)
                quat.append([np.cos(phi, dtype=f32) * sh, 0.0, np.sin(phi, dtype=f32) * sh,
                             np.cos(f32(0.5) * ang, dtype=f32)])
                pos.append([f32(-3.0) + f32(1.2) * f32(ix) + jx, f32(12.0) + f32(2.8) * f32(iy) + jy,
                            f32(11.0) + f32(1.2) * f32(iz) + jz])
    n = len(pos)
    sb.add(np.asarray(pos, np.float32), np.asarray(quat, np.float32), np.full((n, 3), 0.5), SHAPE_BOX, DYN, 5.0,
           friction=0.6, restitution=0.0)
    return sb.build()


SCENES = {1: scene_1, 2: scene_2, 3: scene_3, 4: scene_4, 5: scene_5, 6: scene_6, 7: scene_7}


def reference_scene(k: int) -> dict:
    """Scene k (1..7) of the reference's SceneManager, as a scene dict."""
    if k not in SCENES:
        raise ValueError(f"the reference has scenes 1..7, not {k}")
    return SCENES[k]()
