"""GPU tests of the render feed: per-body 3x4 transforms (world = R local + t) against the
quaternions and positions read back, and the contact points of the last substep against the
step's contact count."""
import numpy as np
import pytest

import beatbox as bb
from beatbox import scenes

pytestmark = pytest.mark.gpu


def rotate(q, v):
    """Rotate v by the unit quaternion q = (x, y, z, w): v + 2 w (u x v) + 2 u x (u x v)."""
    u, w = q[..., :3], q[..., 3:4]
    c = np.cross(u, v)
    return v + 2 * w * c + 2 * np.cross(u, c)


def test_transforms_match_state():
    sc = scenes.box_grid(n_side=6, layers=3)
    w = bb.world_from_scene(sc, params=bb.make_params(solver=bb.SOLVER_PGS_SOFT, quirks=bb.QUIRKS_PHYSICAL))
    for _ in range(20):
        w.step(1 / 60, 2)
    T = w.read_transforms()
    st = w.read_state()
    q = st["quat"].astype(np.float64)
    assert T.shape == (w.n, 3, 4)
    assert np.allclose(T[:, :, 3], st["pos"], atol=0)
    for axis in range(3):
        e = np.zeros((w.n, 3))
        e[:, axis] = 1.0
        assert np.allclose(T[:, :, axis], rotate(q, e), atol=2e-6)
    assert bb.load_library().bb_transforms_device(w.h) is not None
    w.close()


def test_contact_points_cover_the_last_substep():
    sc = scenes.pyramids(n_pyramids=2, boxes_per=100, gap=-0.002)
    w = bb.world_from_scene(sc, params=bb.make_params(solver=bb.SOLVER_PGS_SOFT, quirks=bb.QUIRKS_PHYSICAL))
    w.step(1 / 60, 1)
    pts = w.read_contact_points()
    stats = w.stats()
    assert len(pts) == stats["contact_count"] > 0
    assert np.isfinite(pts).all() and (pts[:, 3] <= 0.01).all()
    w.close()
