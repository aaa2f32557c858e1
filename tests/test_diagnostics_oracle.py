"""The diagnostics oracle (oracle/diagnostics.py) on cases with known answers (no GPU)."""
import numpy as np

from oracle import diagnostics as od


def test_vorticity_of_linear_fields_is_exact():
    x, y, z = np.meshgrid(np.arange(9), np.arange(7), np.arange(5), indexing="ij")
    # u = (0.5 y + 0.25 z, 2 x - z, 0.75 y + x): curl = (0.75 + 1, 0.25 - 1, 2 - 0.5)
    u = np.stack([0.5 * y + 0.25 * z, 2.0 * x - 1.0 * z, 0.75 * y + 1.0 * x]).astype(np.float32)
    assert np.unique(od.vorticity_3d(u, 0, 1.0)).tolist() == [1.75]
    assert np.unique(od.vorticity_3d(u, 1, 1.0)).tolist() == [-0.75]
    assert np.unique(od.vorticity_3d(u, 2, 1.0)).tolist() == [1.5]
    assert np.unique(od.vorticity_2d(u[:2, :, :, 0], 0.5)).tolist() == [3.0]


def test_velocity_rgb_maps_to_unit_range():
    u = np.array([[[0.05, -0.2]], [[0.0, 0.1]]], np.float32)  # (2, 1, 2)
    rgb = od.velocity_rgb(u, 0.1)
    np.testing.assert_allclose(rgb[0, 0], [0.5, 0.75, 0.5], rtol=1e-6)
    np.testing.assert_allclose(rgb[0, 1], [1.0, 0.0, 1.0], rtol=1e-6)


def test_projection_rules():
    u = np.zeros((3, 4, 4, 6), np.float32)
    u[0, 1, 1, 1], u[0, 1, 1, 3] = 0.3, 0.2  # two moving cells in the column (1, 1)
    flag = np.zeros((4, 4, 6), np.int32)
    flag[1, 1, 4] = od.ML_WALL
    u[0, 1, 1, 4] = 9.0  # a wall cell is skipped
    assert od.projection(u, 2, 0, 1.0, flag)[1, 1] == np.float32(0.3)  # maximum
    assert od.projection(u, 2, 1, 1.0, flag)[1, 1] == np.float32(0.2)  # first from the top
    assert od.projection(u, 2, 0, 1.0, flag)[0, 0] == 0.0


def test_polygon_mask_of_a_square():
    sq = np.array([[[2.0, 2.0], [6.0, 2.0], [6.0, 6.0], [2.0, 6.0]]], np.float32)
    m = od.solid_mask_2d(9, 9, sq, np.array([4]), np.array([[4.0, 4.0]]), np.array([1.0 / 9]),
                         np.array([100.0]), 0.5)
    assert m[4, 4] and m[3, 5] and m[2, 4]  # inside, and on the outline
    assert not m[0, 0] and not m[7, 4]


def test_mesh_queries_on_a_triangle_and_a_closed_tetrahedron():
    tri = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)
    assert od.ray_any_hit(tri, np.array([0.2, 0.2, 1.0], np.float32), np.array([0, 0, -1], np.float32), 2.0)
    assert not od.ray_any_hit(tri, np.array([0.2, 0.2, 1.0], np.float32), np.array([0, 0, -1], np.float32), 0.5)
    assert not od.ray_any_hit(tri, np.array([0.8, 0.8, 1.0], np.float32), np.array([0, 0, -1], np.float32), 2.0)
    np.testing.assert_allclose(od._tri_dist2(tri, np.array([0.2, 0.2, 0.5], np.float32)), [0.25], rtol=1e-6)
    np.testing.assert_allclose(od._tri_dist2(tri, np.array([2.0, 0.0, 0.0], np.float32)), [1.0], rtol=1e-6)
    v = np.array([[0, 0, 0], [3, 0, 0], [0, 3, 0], [0, 0, 3]], np.float32)
    tet = v[[[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]]]
    assert od._crossings(tet, np.array([0.5, 0.5, 0.5], np.float32)) % 2 == 1
    assert od._crossings(tet, np.array([2.5, 2.5, 2.5], np.float32)) % 2 == 0
