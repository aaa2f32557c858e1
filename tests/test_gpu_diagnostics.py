"""Field diagnostics on the GPU (openhomelbm_b200.diagnostics, hl_d2q9_image / hl_d3q27_image)
against the oracle's numpy restatement of the reference's display kernels (oracle/diagnostics.py).

Images computed from velocities (|u|, velocity RGB, vorticity slices and projections) must
equal the oracle's binary32 values exactly (same operations, same order, no contraction); the
solid overlays (polygon inside / within a thickness, mesh inside / within a thickness, mesh
silhouettes) must mark the same pixels.
"""
import numpy as np
import pytest
import torch

from oracle import diagnostics as od

pytestmark = pytest.mark.gpu


def _world2d(storage):
    from openhomelbm_b200.batching import capsule_polygon
    from openhomelbm_b200.lbm import LBM_Solver

    s = LBM_Solver(70, 40, solid_num=2, storage=storage, u_scale=0.05, s_scale=1e-3, use_graph=False)
    f = s.flows[0]
    f.vis_shear = 0.02
    f.bc_type = [0, 1, 1, 1]
    f.bc_value = np.array([[0.04, 0.0], [0, 0], [0, 0], [0, 0]], np.float32)
    f.configure_solid(0, capsule_polygon(4.0, 4.0), (22.3, 19.6), angle=0.3, scale=1.0 / 70)
    f.configure_solid(1, capsule_polygon(3.0, 2.5), (47.1, 21.2), angle=-0.7, scale=1.0 / 70)
    for _ in range(30):
        f.solid_position[0, 1] += 0.02
        s.step()
    torch.cuda.synchronize()
    return s, f


def _u2(f):
    return f.decoded()[1:3].float().cpu().numpy()


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_2d_images_match_oracle(storage):
    from openhomelbm_b200 import diagnostics as dg

    s, f = _world2d(storage)
    u = _u2(f)
    np.testing.assert_array_equal(dg.get_u_img(f).cpu().numpy(), od.u_img(u))
    np.testing.assert_array_equal(dg.get_velocity_rgb(f, 0.06).cpu().numpy(), od.velocity_rgb(u, 0.06))
    vort = od.vorticity_2d(u, np.float32(f.grid_length))
    np.testing.assert_array_equal(dg.get_vorticity_img(f).cpu().numpy(), vort)
    mask = od.solid_mask_2d(f.nx, f.ny, f.solid_line_transformed.cpu().numpy(), f.solid_line_num.cpu().numpy(),
                            f.solid_position.cpu().numpy(), f.solid_scale.cpu().numpy(),
                            f.solid_max_radius.cpu().numpy(), 1.5)
    assert 50 < mask.sum() < mask.size // 2
    img = dg.get_vorticity_with_solid_img(f, 1.5).cpu().numpy()
    np.testing.assert_array_equal(img, np.where(mask, od.SOLID_MARK, vort))
    np.testing.assert_array_equal(dg.get_solid_boundary_img(f, 1.5).cpu().numpy(), mask.astype(np.float32))


def _world3d():
    from openhomelbm_b200.lbm3d import LBM_Solver3D
    from openhomelbm_b200.serving import ellipsoid_mesh

    s = LBM_Solver3D(30, 24, 20, solid_num=1, use_graph=False)
    f = s.flows[0]
    f.vis_shear = 0.02
    f.bc_type = [0, 1, 1, 1, 1, 1]
    f.bc_value = np.array([[0.03, 0.0, 0.0]] + [[0, 0, 0]] * 5, np.float32)
    s.create_solid_from_mesh(0, ellipsoid_mesh(6.0, 3.0, 2.5, 16, 9), lbm_position=(9.3, 11.7, 9.6),
                             lbm_scale=1.0 / 30, init_quaternion=(0.96, 0.0, 0.1, 0.26))
    for _ in range(12):
        s.step()
    torch.cuda.synchronize()
    return s, f


def test_3d_slices_and_projections_match_oracle():
    from openhomelbm_b200 import diagnostics as dg

    s, f = _world3d()
    u = f.decoded()[1:4].float().cpu().numpy()
    h = np.float32(f.grid_length)
    mag = np.sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
    np.testing.assert_array_equal(dg.get_u_img_xy_3d(f, 7).cpu().numpy(), od.plane(mag, 2, 7))
    np.testing.assert_array_equal(dg.get_u_img_yz_3d(f, 11).cpu().numpy(), od.plane(mag, 0, 11))
    np.testing.assert_array_equal(dg.get_vorticity_xy_3d(f, 9).cpu().numpy(), od.plane(od.vorticity_3d(u, 2, h), 2, 9))
    np.testing.assert_array_equal(dg.get_vorticity_yz_3d(f, 4).cpu().numpy(), od.plane(od.vorticity_3d(u, 0, h), 0, 4))

    tri_offset = s._tri_offset.cpu().numpy()
    tris = s._tris.cpu().numpy()
    xf = s.mesh_transforms_all[0].cpu().numpy()
    sc = s.mesh_scale_sizes_all[0].cpu().numpy()
    flag = f.flag.cpu().numpy()
    shape = (f.nx, f.ny, f.nz)
    for axis, fn in ((2, dg.get_vorticity_xy_with_solid_3d), (0, dg.get_vorticity_yz_with_solid_3d)):
        idx = 9 if axis == 2 else 10
        mask = od.solid_plane_mask(shape, axis, idx, tri_offset, tris, xf, sc, 1.0, flag)
        assert mask.sum() > 10
        ref = np.where(mask, od.SOLID_MARK, od.plane(od.vorticity_3d(u, axis, h), axis, idx))
        np.testing.assert_array_equal(fn(f, idx, 1.0).cpu().numpy(), ref)

    cases = [(dg.get_u_projection_topdown_3d, 2, 1), (dg.get_u_projection_max_topdown_3d, 2, 0),
             (dg.get_vorticity_projection_topdown_3d, 2, 2), (dg.get_u_projection_side_3d, 0, 0),
             (dg.get_u_projection_front_3d, 1, 0), (dg.get_vorticity_projection_side_3d, 0, 2),
             (dg.get_vorticity_projection_front_3d, 1, 2)]
    sil = {a: od.silhouette(shape, a, tri_offset, tris, xf, sc) for a in (0, 1, 2)}
    for fn, axis, kind in cases:
        assert sil[axis].sum() > 10
        ref = np.where(sil[axis], od.SOLID_MARK, od.projection(u, axis, kind, h, flag))
        np.testing.assert_array_equal(fn(f).cpu().numpy(), ref, err_msg=fn.__name__)


def test_image_entry_points_reject_bad_arguments():
    from openhomelbm_b200 import _lib
    from openhomelbm_b200 import diagnostics as dg

    s, f = _world2d("float32")
    with pytest.raises(ValueError):
        dg.get_velocity_rgb(f, 0.0)
    out = torch.zeros(4, device=f.device)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib().hl_d2q9_image(dg._world2d(f), 7, 0.0, 0.0, None, 0.0, out.data_ptr(), _lib.stream_ptr()))
    s3, f3 = _world3d()
    with pytest.raises(ValueError):
        dg.get_u_img_xy_3d(f3, f3.nz)  # slice outside the grid


@pytest.mark.parametrize("slice_axis,color_axis,margin", [(2, 2, 0), (0, 1, 2), (1, 0, 1)])
def test_live_slices_histogram_and_rgba_match_oracle(slice_axis, color_axis, margin):
    from openhomelbm_b200 import diagnostics as dg

    s, f = _world3d()
    u = f.decoded()[1:4].float().cpu().numpy()
    n = (f.nx, f.ny, f.nz)
    inplane = [a for a in range(3) if a != slice_axis]
    stride = 2
    W, H = n[inplane[0]] // stride + 2, n[inplane[1]] // stride + 2  # samples past the edge clamp
    # the flow (started at rest, inflow at x = 0) has reached the first few x planes only;
    # the last position lies outside the grid
    positions = [3, n[slice_axis] // 2, n[slice_axis] - 1, n[slice_axis] + 3]
    pos = torch.tensor(positions, dtype=torch.int32, device=f.device)
    values = torch.full((len(positions) * W * H,), 7.0, device=f.device)
    hist = torch.ones(256, dtype=torch.int32, device=f.device)
    dg.clear_live_histogram(hist)
    dg.extract_live_vorticity_slices(f, pos, values, hist, W, H, stride, slice_axis, color_axis, margin, 1)
    ref = od.live_slices(u, positions, W, H, stride, slice_axis, color_axis, margin)
    np.testing.assert_array_equal(values.cpu().numpy(), ref)
    h_ref, ambiguous = od.live_histogram(ref)
    h = hist.cpu().numpy()
    assert h_ref.sum() > 20 and h.sum() == h_ref.sum()
    assert np.abs(h - h_ref).sum() <= 2 * ambiguous
    vmax = dg.vmax_from_histogram(h, 98.0)
    rgba = torch.zeros(values.numel() * 4, dtype=torch.uint8, device=f.device)
    dg.live_vorticity_to_rgba(values, rgba, vmax, 0.8)
    np.testing.assert_array_equal(rgba.cpu().numpy().reshape(-1, 4), od.live_rgba(ref, vmax, 0.8))
    # without collecting, the histogram is left alone
    before = hist.clone()
    dg.extract_live_vorticity_slices(f, pos, values, hist, W, H, stride, slice_axis, color_axis, margin, 0)
    assert torch.equal(hist, before)


def test_2d_realtime_rgba_and_controls():
    """The 2D realtime tool's GPU kernels: u_img to RGBA in the three render modes, the local
    force field, and the boundary-velocity and prescribed-motion controls."""
    from openhomelbm_b200 import diagnostics as dg
    from openhomelbm_b200.lbm import controls

    s, f = _world2d("float32")
    fills = ((0, dg.get_u_img), (1, lambda fl: dg.get_vorticity_with_solid_img(fl, 1.5)),
             (2, lambda fl: dg.get_solid_boundary_img(fl, 1.5)))
    for mode, fill in fills:
        img = fill(f).cpu().numpy()
        vmax = {0: 0.06, 1: float(np.abs(img[img < 999]).max()) * 0.5, 2: 1.0}[mode]
        out = torch.zeros((f.ny, f.nx, 4), dtype=torch.uint8, device=f.device)
        dg.lbm_uimg_to_rgba(f, out, mode, vmax)
        np.testing.assert_array_equal(out.cpu().numpy(), od.uimg_rgba(img, mode, vmax))
        if mode == 1:
            assert (out.cpu().numpy()[..., 0] == 200).sum() > 20  # the solid marks
    controls.set_local_force(s.flows, 30.5, 20.0, 6.0, 4.0, 1e-5, -2e-5)
    fx, fy = od.local_force(f.nx, f.ny, 30.5, 20.0, 6.0, 4.0, 1e-5, -2e-5)
    np.testing.assert_array_equal(f.force[0].cpu().numpy(), fx)
    np.testing.assert_array_equal(f.force[1].cpu().numpy(), fy)
    assert f.use_force and (fx > 0).sum() > 50
    controls.set_boundary_velocity(s.flows, 0, 0.03, 0.01)
    np.testing.assert_allclose(f.bc_value[0], [0.03, 0.01], rtol=1e-6)
    p0, a0 = f.solid_position[1].clone(), float(f.solid_angle[1])
    controls.advance_prescribed_solid_motion(s.flows, 1, 0.5, -0.25, 0.1)
    torch.testing.assert_close(f.solid_position[1], p0 + torch.tensor([0.5, -0.25], device=f.device))
    assert abs(float(f.solid_angle[1]) - (a0 + 0.1)) < 1e-6
    s.step()  # forced, new inflow, moved solid
    torch.cuda.synchronize()
    assert torch.isfinite(f.decoded()).all()
    with pytest.raises(ValueError):
        controls.set_boundary_velocity(s.flows, 4, 0.0, 0.0)
    with pytest.raises(ValueError):
        dg.lbm_uimg_to_rgba(f, torch.zeros((f.nx, f.ny, 4), dtype=torch.uint8, device=f.device), 0, 0.1)
