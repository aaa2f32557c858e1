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


def test_live_slices_oracle_on_linear_fields():
    """The live view's vorticity of u = (a z, b x, c y) is (c, a, b) everywhere, border samples
    (one-sided, divided by the clamped span) and clamped in-plane samples included; a position
    outside the grid gives zeros; the margin zeroes the cells near a face."""
    n = (6, 7, 8)
    x, y, z = np.meshgrid(*(np.arange(k, dtype=np.float32) for k in n), indexing="ij")
    u = np.stack([0.5 * z, 0.25 * x, 0.125 * y]).astype(np.float32)  # curl = (0.125, 0.5, 0.25)
    for slice_axis in range(3):
        for color_axis, want in enumerate((0.125, 0.5, 0.25)):
            v = od.live_slices(u, [1, n[slice_axis] - 1, n[slice_axis]], 5, 6, 2, slice_axis, color_axis, 0)
            v = v.reshape(3, 6, 5)
            np.testing.assert_array_equal(v[:2], np.float32(want))
            np.testing.assert_array_equal(v[2], 0)
    m = od.live_slices(u, [3], 5, 6, 1, 2, 2, 1).reshape(6, 5)  # z = 3, x = p, y = q
    np.testing.assert_array_equal(m[1:6, 1:5], np.float32(0.25))
    assert (m[0] == 0).all() and (m[:, 0] == 0).all()


def test_live_histogram_rgba_and_vmax():
    from openhomelbm_b200 import diagnostics as dg

    vals = np.array([0, 1e-9, 1e-8 * 1.01, 3e-4, -3e-4, 0.5, 2.0], np.float32)
    h, amb = od.live_histogram(vals)
    assert h.sum() == 5 and h[-1] == 1 and amb == 0  # 0.5 and 2 (clamped) share the top bins
    assert h[int(np.clip((np.log(3e-4) + 18.420680743952367) / 18.420680743952367, 0, 0.999999) * 256)] == 2
    assert od.live_histogram(np.array([1e-4], np.float32))[1] == 1  # log 1e-4 is a bin edge
    rgba = od.live_rgba(np.array([-3, -0.5, 0, 0.5, 3], np.float32), 1.0, 0.5)
    np.testing.assert_array_equal(rgba[:, 3], 127)
    np.testing.assert_array_equal(rgba[[0, 2, 4], :3], [[0, 0, 255], [255, 255, 255], [255, 0, 0]])
    counts = np.zeros(256, np.int64)
    counts[100] = 10
    want = np.exp(-18.420680743952367 * (1 - 100.5 / 256))
    assert abs(dg.vmax_from_histogram(counts, 98.0) - want) < 1e-12 * want
    assert dg.vmax_from_histogram(np.zeros(256), 98.0) == 1e-6
    assert dg.vmax_from_histogram(counts, 98.0, previous=10 * want) == 9.6 * want
    counts[200] = 1  # the 98th percentile of 11 counts is the 11th: bin 200
    assert abs(dg.vmax_from_histogram(counts, 98.0) - np.exp(-18.420680743952367 * (1 - 200.5 / 256))) < 1e-9


def test_2d_realtime_oracle_maps():
    img = np.array([[0.0, 0.5], [1.0, 2.0]], np.float32)  # (nx, ny)
    out = od.uimg_rgba(img, 0, 1.0)
    assert out.shape == (2, 2, 4) and (out[..., 3] == 255).all()
    np.testing.assert_array_equal(out[0, 0, :3], [0, 0, 60])      # x 0, y 0: zero
    np.testing.assert_array_equal(out[1, 0, :3], [127, 45, 30])   # x 0, y 1: half
    np.testing.assert_array_equal(out[0, 1, :3], [255, 180, 0])   # x 1, y 0: full
    v = od.uimg_rgba(np.array([[-1.0, 1000.0], [0.0, 1.0]], np.float32), 1, 1.0)
    # (y, x) order: (0, 0) -1 blue, (0, 1) 0 white, (1, 0) the solid mark grey, (1, 1) 1 red
    np.testing.assert_array_equal(v[:, :, :3].reshape(-1, 3), [[0, 0, 255], [255, 255, 255], [200, 200, 200],
                                                               [255, 0, 0]])
    np.testing.assert_array_equal(od.uimg_rgba(np.array([[0.0, 0.25]], np.float32), 2, 1.0)[:, 0, 0], [255, 191])
    fx, fy = od.local_force(5, 5, 2, 2, 2, 2, 1.0, -2.0)
    assert fx[2, 2] == 1.0 and fy[2, 2] == -2.0 and fx[0, 0] == 0 and fx[2, 3] == np.float32(0.75)


# --------------------------------------------------------------------------- pinned to the reference
def _golden():
    from conftest import load_golden

    return load_golden("diagnostics")


def test_2d_display_kernels_match_reference_fixture():
    """oracle/diagnostics.py against the reference's own 2D display kernels (get_u_img,
    get_velocity_rgb, get_vorticity_img, get_vorticity_with_solid_img, get_solid_boundary_img,
    envs/lbm/lbm_func.py:163-319, 804-866) and the 2D tool's kernels (lbm_uimg_to_rgba_kernel,
    set_local_force_kernel, tools/lbm2d_realtime_control.py:144-157, 417-464), run under the
    Warp emulator by tests/golden/make_golden.py: bit for bit."""
    g = _golden()
    u = g["u2"]
    nx, ny = u.shape[1:]
    np.testing.assert_array_equal(od.u_img(u), g["u_img"])
    np.testing.assert_array_equal(od.velocity_rgb(u, 0.05), g["velocity_rgb"])
    vort = od.vorticity_2d(u, g["grid_length2"])
    np.testing.assert_array_equal(vort, g["vorticity2"])
    mask = od.solid_mask_2d(nx, ny, g["line_tf2"], g["line_num2"], g["position2"], g["scale2"], g["max_radius2"], 1.3)
    assert 20 < mask.sum() < mask.size // 2
    np.testing.assert_array_equal(np.where(mask, od.SOLID_MARK, vort), g["vorticity2_solid"])
    np.testing.assert_array_equal(mask.astype(np.float32), g["solid_boundary2"])
    for mode, key, vmax in ((0, "u_img", 0.06), (1, "vorticity2", 0.02), (2, "solid_boundary2", 1.0)):
        np.testing.assert_array_equal(od.uimg_rgba(g[key], mode, vmax), g[f"uimg_rgba_{mode}"], err_msg=str(mode))
    fx, fy = od.local_force(nx, ny, *g["local_force_args"])
    np.testing.assert_array_equal(np.stack([fx, fy]), g["local_force"])


def test_3d_display_kernels_match_reference_fixture():
    """The 3D slices and projections, silhouettes of a scaled, rotated mesh included
    (envs/lbm3d/lbm_func_3d.py:320-362, 753-842, 990-1313), against the reference's kernels
    under the emulator, bit for bit. The ray queries of the silhouettes are Warp's native
    mesh_query_ray in the reference and a Moller-Trumbore restatement in the emulator and here."""
    g = _golden()
    u = g["u3"]
    h = g["grid_length3"]
    flag = g["flag3"]
    mag = np.sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
    np.testing.assert_array_equal(od.plane(mag, 2, 6), g["u_xy_6"])
    np.testing.assert_array_equal(od.plane(mag, 0, 5), g["u_yz_5"])
    np.testing.assert_array_equal(od.plane(od.vorticity_3d(u, 2, h), 2, 3), g["vort_xy_3"])
    np.testing.assert_array_equal(od.plane(od.vorticity_3d(u, 0, h), 0, 9), g["vort_yz_9"])
    tris = g["mesh_vertices"][g["mesh_faces"]].astype(np.float32)
    tri_offset = np.array([0, len(tris)], np.int32)
    xf, sc = g["mesh_transform"][None], g["mesh_scale"][None]
    shape = u.shape[1:]
    sil = {a: od.silhouette(shape, a, tri_offset, tris, xf, sc) for a in (0, 1, 2)}
    for name, axis, kind in (("get_u_projection_topdown_3d", 2, 1), ("get_u_projection_max_topdown_3d", 2, 0),
                             ("get_vorticity_projection_topdown_3d", 2, 2), ("get_u_projection_side_3d", 0, 0),
                             ("get_u_projection_front_3d", 1, 0), ("get_vorticity_projection_side_3d", 0, 2),
                             ("get_vorticity_projection_front_3d", 1, 2)):
        assert sil[axis].sum() > 5
        ref = np.where(sil[axis], od.SOLID_MARK, od.projection(u, axis, kind, h, flag))
        np.testing.assert_array_equal(ref, g[name], err_msg=name)


def test_live_view_kernels_match_reference_fixture():
    """The live 3D view's slice stack, histogram and colour map
    (tools/lbm3d_realtime_control.py:68-182) against the reference's kernels under the emulator:
    values and RGBA bytes bit for bit; histogram counts equal except for values within 1e-4 of a
    bin edge (the emulator's binary32 logarithm, the oracle's binary64 one)."""
    g = _golden()
    u = g["u3"]
    assert int(g["live_bins"]) == od.LIVE_BINS
    k = 0
    while f"live{k}_args" in g:
        slice_axis, color_axis, stride, margin, pw, ph = (int(v) for v in g[f"live{k}_args"])
        vals = od.live_slices(u, g[f"live{k}_positions"], pw, ph, stride, slice_axis, color_axis, margin)
        np.testing.assert_array_equal(vals, g[f"live{k}_values"], err_msg=str(k))
        hist, near_edge = od.live_histogram(vals)
        assert np.abs(hist - g[f"live{k}_hist"]).sum() <= 2 * near_edge, k
        np.testing.assert_array_equal(od.live_rgba(vals, 0.05, 0.8).reshape(-1), g[f"live{k}_rgba"], err_msg=str(k))
        k += 1
    assert k == 3
