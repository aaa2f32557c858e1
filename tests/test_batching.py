"""Host side of the batching form (no GPU): the tile work-list of hl_d2q9_tile_list, the
capsule outline, the swimmer's travelling-wave kinematics and the seeded world sizes."""
import math

import numpy as np
import pytest

from openhomelbm_b200 import batching


def test_tile_shapes_listed():
    shapes = batching.tile_shapes()
    assert (16, 32) in shapes and len(shapes) == len(set(shapes)) >= 4
    assert all(tx >= 1 and ty >= 30 for tx, ty in shapes)
    assert (64, 30) in shapes  # strips: a warp per 30-row tile


@pytest.mark.parametrize("shape", [(8, 32), (16, 64), (8, 128), (64, 30)])
def test_tile_list_covers_every_cell_once(shape):
    sizes = [(37, 29), (130, 70), (64, 64), (1, 1)][:3] + [(300, 129)]
    nx, ny = [s[0] for s in sizes], [s[1] for s in sizes]
    t = batching.tile_list(nx, ny, shape)
    assert t.dtype == np.int32 and t.shape[1] == 4 and (t[:, 3] == 0).all()
    assert (np.diff(t[:, 0]) >= 0).all()  # world-major
    for w, (a, b) in enumerate(sizes):
        cover = np.zeros((a, b), np.int32)
        for _, x0, y0, _ in t[t[:, 0] == w]:
            cover[x0:x0 + shape[0], y0:y0 + shape[1]] += 1
        assert (cover == 1).all()
        assert (t[:, 0] == w).sum() == math.ceil(a / shape[0]) * math.ceil(b / shape[1])


def test_tile_list_rejects_bad_input():
    with pytest.raises(ValueError):
        batching.tile_list([64], [64], (7, 32))
    with pytest.raises(ValueError):
        batching.tile_list([2], [64], (8, 32))


def test_capsule_polygon_is_a_stadium():
    p = batching.capsule_polygon(4.0, 4.0)
    assert p.shape == (26, 2)
    np.testing.assert_allclose(p[:, 0].min(), -8.0, atol=1e-5)
    np.testing.assert_allclose(p[:, 0].max(), 8.0, atol=1e-5)
    np.testing.assert_allclose(np.abs(p[:, 1]).max(), 4.0, atol=1e-5)
    # counter-clockwise: positive signed area, a little below the stadium's (2 a) (2 r) + pi r^2
    x, y = p[:, 0].astype(np.float64), p[:, 1].astype(np.float64)
    area = 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)
    assert 0.97 * (64 + math.pi * 16) < area < 64 + math.pi * 16


def test_capsule_chain_follows_the_travelling_wave():
    ch = batching.CapsuleChain(head=(100.0, 50.0), freq=0.01)
    t = np.array([0.0, 0.3, 7.25])
    pos, ang = ch.poses_at(t)
    assert pos.shape == (3, 8, 2) and ang.shape == (3, 8)
    s = np.linspace(0, 64, 9)
    for j, tj in enumerate(t):
        y = ch.centreline(s, np.full_like(s, tj))
        np.testing.assert_allclose(pos[j, :, 0], 100.0 + 0.5 * (s[1:] + s[:-1]))
        np.testing.assert_allclose(pos[j, :, 1], 50.0 + 0.5 * (y[1:] + y[:-1]))
        np.testing.assert_allclose(np.tan(ang[j]), (y[1:] - y[:-1]) / 8.0, rtol=1e-12, atol=1e-12)
    # amplitude envelope: 0.02 L at the head, 0.1 L at the tail
    np.testing.assert_allclose(ch.centreline(np.array([0.0]), np.array([-0.25 / 0.01]))[0], 0.02 * 64 * np.sin(
        2 * np.pi * 0.25), rtol=1e-12)
    np.testing.assert_allclose(ch.centreline(np.array([64.0]), np.array([0.75 / 0.01]))[0], 0.1 * 64 * np.sin(
        2 * np.pi * (1 - 0.75)), rtol=1e-12)


def test_swimmer_wall_speed_stays_low_mach():
    # highest frequency, 8 substeps: the tail moves at most 2 pi f A_tail / 8 per LBM step
    ch = batching.CapsuleChain(head=(0.0, 0.0), freq=0.01)
    t = np.linspace(0, 100, 801)  # one sample per LBM substep
    pos, _ = ch.poses_at(t)
    v = np.abs(np.diff(pos[:, :, 1], axis=0)).max()
    assert v <= 2 * np.pi * 0.01 * 6.4 / 8 * 1.01
    assert v < 0.06


def test_batch_sizes_are_seeded_log_uniform():
    a = batching.batch_sizes(64, seed=0)
    assert a == batching.batch_sizes(64, seed=0) and a != batching.batch_sizes(64, seed=1)
    nx = np.array([s[0] for s in a])
    ny = np.array([s[1] for s in a])
    assert nx.min() >= 256 and nx.max() <= 1024 and ny.min() >= 128 and ny.max() <= 512
    specs = batching.swimmer_specs(64, seed=0)
    assert [(s.nx, s.ny) for s in specs] == a
    f = np.array([s.chain.freq for s in specs])
    assert f.min() >= 0.002 and f.max() <= 0.01


def test_chain_poses_equal_per_chain_poses():
    specs = batching.swimmer_specs(6, seed=2)
    t = np.array([0.125, 3.5, 17.0])
    pos, ang = batching.chain_poses([s.chain for s in specs], t)
    assert pos.shape == (3, 6, 8, 2) and ang.shape == (3, 6, 8)
    for w, s in enumerate(specs):
        p, a = s.chain.poses_at(t)
        np.testing.assert_allclose(pos[:, w], p, rtol=0, atol=1e-12)
        np.testing.assert_allclose(ang[:, w], a, rtol=0, atol=1e-12)
    with pytest.raises(ValueError):
        batching.chain_poses([specs[0].chain, batching.CapsuleChain(head=(0, 0), freq=0.01, length=32.0)], t)
