"""The masked world resets against the reference's own kernels (tests/golden/reset.npz, made by
tests/golden/make_golden.py from ResetSingleWorldFlow(3D), ResetSingleWorldSolidTransform(3D)
and ResetSingleWorldForces(3D), envs/lbm/lbm_func.py:66-160 and envs/lbm3d/lbm_func_3d.py:86-196,
over three worlds of random state), bit for bit, through the solvers' ``flows_wp``; and the
host-side reads of the drop-in fields (``numpy()`` as on a Warp array).
"""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _solver3d(g):
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    nworld, nsol = g["cur3_before"].shape[0], g["tf3_before"].shape[1]
    nx, ny, nz = g["cur3_before"].shape[2:]
    s = LBM_Solver3D(nx, ny, nz, solid_num=nsol, nworld=nworld, use_graph=False)
    dev = s.device
    for w, f in enumerate(s.flows):
        f.cur.copy_(torch.tensor(g["cur3_before"][w], device=dev))
        f.post.copy_(torch.tensor(g["post3_before"][w], device=dev))
        f.force.copy_(torch.tensor(g["force3_before"][w], device=dev))
        f.mesh_transforms.copy_(torch.tensor(g["tf3_before"][w], device=dev))
        f.mesh_transforms_last.copy_(torch.tensor(g["tf_last3_before"][w], device=dev))
        f.mesh_transforms_initialized.copy_(torch.tensor(g["initialized3_before"][w], device=dev))
        f.solid_force.copy_(torch.tensor(g["solid_force3_before"][w], device=dev))
        f.solid_torque.copy_(torch.tensor(g["solid_torque3_before"][w], device=dev))
    return s


def _check3d(s, g, suffix):
    for w, f in enumerate(s.flows):
        for name, got in (("cur3", f.cur), ("post3", f.post), ("force3", f.force), ("tf3", f.mesh_transforms),
                          ("tf_last3", f.mesh_transforms_last), ("initialized3", f.mesh_transforms_initialized),
                          ("solid_force3", f.solid_force), ("solid_torque3", f.solid_torque)):
            ref = g[f"{name}_{suffix}"][w]
            assert np.array_equal(got.cpu().numpy(), ref), (name, w)


def test_reset_3d_matches_reference_kernels():
    from openhomelbm_b200.lbm3d.lbm_func_3d import (ResetSingleWorldFlow3D, ResetSingleWorldForces3D,
                                                    ResetSingleWorldSolidTransform3D, reset_worlds_masked)

    g = load_golden("reset")
    # the three kernels one by one, as partial_reset launches them, with a host mask
    s = _solver3d(g)
    ResetSingleWorldFlow3D(s.flows_wp, g["mask3"])
    ResetSingleWorldSolidTransform3D(s.flows_wp, g["mask3"])
    ResetSingleWorldForces3D(s.flows_wp, g["mask3"])
    torch.cuda.synchronize()
    _check3d(s, g, "after")
    # all three in one launch, with the mask already on the device
    s = _solver3d(g)
    reset_worlds_masked(s.flows_wp, torch.tensor(g["mask3"], dtype=torch.int32, device=s.device))
    torch.cuda.synchronize()
    _check3d(s, g, "after")


def test_solver_reset_worlds_resets_flow_and_initialized_only():
    """LBM_Solver3D.reset_worlds (lbm_solver_3d.py:367-385): the flow reset plus
    mesh_transforms_initialized = 0; the transforms and loads stay."""
    g = load_golden("reset")
    s = _solver3d(g)
    s.reset_worlds([0, 2])
    torch.cuda.synchronize()
    for w, f in enumerate(s.flows):
        reset = w in (0, 2)
        src = "after" if reset else "before"
        assert np.array_equal(f.cur.cpu().numpy(), g[f"cur3_{src}"][w])
        assert np.array_equal(f.post.cpu().numpy(), g[f"post3_{src}"][w])
        assert np.array_equal(f.force.cpu().numpy(), g[f"force3_{src}"][w])
        assert np.array_equal(f.mesh_transforms.cpu().numpy(), g["tf3_before"][w])
        assert np.array_equal(f.solid_force.cpu().numpy(), g["solid_force3_before"][w])
        assert np.array_equal(f.mesh_transforms_initialized.cpu().numpy(),
                              np.zeros(2, np.int32) if reset else g["initialized3_before"][w])
    with pytest.raises(ValueError):
        s.reset_worlds([3])


def _solver2d(g):
    from openhomelbm_b200.lbm import LBM_Solver

    nworld = g["cur2_before"].shape[0]
    nx, ny = g["cur2_before"].shape[2:]
    nsol = g["solid_line"].shape[0]
    s = LBM_Solver(nx, ny, solid_num=nsol, nworld=nworld, use_graph=False)
    dev = s.device
    for w, f in enumerate(s.flows):
        for sid in range(nsol):
            n = int(g["solid_line_num"][sid])
            f.configure_solid(sid, g["solid_line"][sid, :n], (3.0, 2.0), scale=1.0 / nx)
        assert f.max_segments_per_object == g["line_tf2_before"].shape[2]
        f.cur.copy_(torch.tensor(g["cur2_before"][w], device=dev))
        f.post.copy_(torch.tensor(g["post2_before"][w], device=dev))
        f.force.copy_(torch.tensor(g["force2_before"][w], device=dev))
        f.solid_line_transformed.copy_(torch.tensor(g["line_tf2_before"][w], device=dev))
        f.solid_line_transformed_last.copy_(torch.tensor(g["line_tf_last2_before"][w], device=dev))
        s.solid_loads_all[w].copy_(torch.tensor(g["loads2_before"][w], device=dev))
    return s


def test_reset_2d_matches_reference_kernels():
    from openhomelbm_b200.lbm.lbm_func import (ResetSingleWorldFlow, ResetSingleWorldForces,
                                               ResetSingleWorldSolidTransform)

    g = load_golden("reset")
    s = _solver2d(g)
    ResetSingleWorldFlow(s.flows_wp, g["mask2"])
    ResetSingleWorldSolidTransform(s.flows_wp, g["mask2"])
    ResetSingleWorldForces(s.flows_wp, g["mask2"])
    torch.cuda.synchronize()
    s2 = _solver2d(g)
    s2.reset_worlds_mask(g["mask2"].astype(bool))
    torch.cuda.synchronize()
    for solver in (s, s2):
        for w, f in enumerate(solver.flows):
            for name, got in (("cur2", f.cur), ("post2", f.post), ("force2", f.force),
                              ("line_tf2", f.solid_line_transformed), ("line_tf_last2", f.solid_line_transformed_last),
                              ("loads2", solver.solid_loads_all[w])):
                assert np.array_equal(got.cpu().numpy(), g[f"{name}_after"][w]), (name, w)


def test_fields_read_back_like_warp_arrays():
    """flows[w].<field>.numpy() gives a host copy, as on a Warp array on the GPU
    (envs/lbm/eel/eel_lbm_env.py:126, envs/lbm3d/eel/eel_lbm_env_3d.py:1182)."""
    from openhomelbm_b200.lbm import LBM_Solver
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    s3 = LBM_Solver3D(6, 6, 6, solid_num=2, nworld=2, use_graph=False)
    s3.flows[1].solid_position[1] = torch.tensor([1.0, 2.0, 3.0], device=s3.device)
    p = s3.flows[1].solid_position.numpy()
    assert isinstance(p, np.ndarray) and p.shape == (2, 3) and p[1].tolist() == [1.0, 2.0, 3.0]
    assert s3.flows[0].rho.numpy().shape == (6, 6, 6) and s3.flows[0].u.numpy().shape == (6, 6, 6, 3)
    assert len(s3.flows_wp) == 2 and s3.flows_wp[1] is s3.flows[1]
    s2 = LBM_Solver(8, 6, solid_num=1, nworld=2, use_graph=False)
    assert s2.flows[1].solid_max_radius.numpy().shape == (1,)
    assert s2.flows[0].u.numpy().shape == (8, 6, 2)
    s2.step()  # the views stay usable in a step
    assert np.isfinite(s2.flows[0].rho.numpy()).all()
