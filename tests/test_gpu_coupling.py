"""MuJoCo-Warp coupling kernels on the GPU against the reference's kernels run on the same
random buffers (golden fixture ``coupling``): body-state extraction, pose conversion into the
solids (3D transforms with their last/initialised bookkeeping, 2D yaw), load extraction in
the three forms, and the xfrc_applied fill. Copies and scalings are exact; the pose
conversion and the yaw are compared to 1e-6 (the GPU may fuse the multiply-add, the
reference's binary32 arithmetic rounds twice; atan2 implementations differ in the last bit).
"""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _t(a, dtype=torch.float32):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def test_coupling_3d_matches_reference():
    from openhomelbm_b200 import coupling
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    g = load_golden("coupling")
    nworld, nbody = g["xipos"].shape[:2]
    nsel = len(g["body_ids"])
    body_ids = _t(g["body_ids"], torch.int32)
    pos = torch.zeros((nworld, nsel, 3), device="cuda")
    quat = torch.zeros((nworld, nsel, 4), device="cuda")
    coupling.extract_body_states_3d(_t(g["xipos"]), _t(g["xquat"]), body_ids, pos, quat)
    # (the fixture's pos_out was saved after the generator's two += 0.01 below)
    np.testing.assert_array_equal(pos.cpu().numpy(), g["xipos"][:, g["body_ids"]])
    np.testing.assert_array_equal(quat.cpu().numpy(), g["xquat"][:, g["body_ids"]])
    np.testing.assert_array_equal(quat.cpu().numpy(), g["quat_out"])

    s = LBM_Solver3D(6, 6, 6, solid_num=nsel, nworld=nworld, use_graph=False)
    sids = _t(np.arange(nsel), torch.int32)
    for call in range(2):  # the first call initialises, the second moves current -> last
        coupling.convert_and_update_solid_batch_3d(s, sids, pos, quat, mujoco_origins=_t(g["mj_origin"]),
                                                   lbm_origins=_t(g["lbm_origin"]), scales=_t(g["scales"]))
        got = np.stack([np.stack([s.mesh_transforms_all[w].cpu().numpy(), s.mesh_transforms_last_all[w].cpu().numpy()])
                        for w in range(nworld)])
        np.testing.assert_allclose(got, g["tf_hist"][call], rtol=1e-6, atol=1e-6)
        assert (s.mesh_transforms_initialized_all.cpu().numpy() == 1).all()
        pos += 0.01
    np.testing.assert_allclose(s.solid_position_all.cpu().numpy(), g["tf_hist"][1][:, 0, :, :3], rtol=1e-6)
    np.testing.assert_array_equal(s.solid_quaternion_all.cpu().numpy(), g["quat_out"])

    s.solid_force_all.copy_(_t(g["solid_force3"]))
    s.solid_torque_all.copy_(_t(g["solid_torque3"]))
    fo = torch.zeros((nworld, nsel, 3), device="cuda")
    to = torch.zeros((nworld, nsel, 3), device="cuda")
    coupling.extract_forces_torques_physical_3d(s, sids, float(g["force_conv"]), float(g["torque_conv"]), fo, to)
    np.testing.assert_array_equal(fo.cpu().numpy(), g["forces3"])
    np.testing.assert_array_equal(to.cpu().numpy(), g["torques3"])
    xfrc = torch.zeros((nworld, nbody, 6), device="cuda")
    coupling.fill_xfrc_3d_kernel(xfrc, body_ids, fo, to)
    np.testing.assert_array_equal(xfrc.cpu().numpy(), g["xfrc3"])

    # /scale form (extract_forces_torques_batch_3d)
    coupling.extract_forces_torques_batch_3d(s, sids, _t(g["scales"]), fo, to)
    sc = g["scales"][None, :, None]
    np.testing.assert_allclose(fo.cpu().numpy(), g["solid_force3"] / sc, rtol=1e-6)
    np.testing.assert_allclose(to.cpu().numpy(), g["solid_torque3"] / (sc * sc), rtol=1e-6)


def test_coupling_2d_matches_reference():
    from openhomelbm_b200 import coupling
    from openhomelbm_b200.lbm import LBM_Solver

    g = load_golden("coupling")
    nworld, nbody = g["xipos"].shape[:2]
    nsel = len(g["body_ids"])
    s = LBM_Solver(6, 6, solid_num=nsel, nworld=nworld, use_graph=False)
    sids = _t(np.arange(nsel), torch.int32)
    coupling.convert_and_update_solid_batch_2d(s, sids, _t(g["pos_after"]), _t(g["quat_out"]),
                                               mujoco_origins=_t(g["mj_origin"][:, :2]),
                                               lbm_origins=_t(g["lbm_origin"][:, :2]), scales=_t(g["scales"]))
    np.testing.assert_allclose(s.solid_position_all.cpu().numpy(), g["solid_position2"], rtol=1e-6)
    np.testing.assert_allclose(s.solid_angle_all.cpu().numpy(), g["solid_angle2"], rtol=0, atol=2e-6)
    # the solver's own views see the batched values
    np.testing.assert_array_equal(s.flows[1].solid_angle.cpu().numpy(), s.solid_angle_all[1].cpu().numpy())

    s.solid_loads_all.copy_(_t(g["loads2"]))
    fo = torch.zeros((nworld, nsel, 3), device="cuda")
    to = torch.zeros((nworld, nsel, 3), device="cuda")
    coupling.extract_forces_torques_batch(s, sids, _t(g["scales"]), fo, to)
    np.testing.assert_array_equal(fo.cpu().numpy(), g["forces2"])
    np.testing.assert_array_equal(to.cpu().numpy(), g["torques2"])
    np.testing.assert_array_equal(s.flows[0].torque.cpu().numpy(), g["loads2"][0, 2])
    xfrc = torch.zeros((nworld, nbody, 6), device="cuda")
    coupling.fill_xfrc_kernel(xfrc, _t(g["body_ids"], torch.int32), fo, to)
    np.testing.assert_array_equal(xfrc.cpu().numpy(), g["xfrc2"])


def test_coupling_rejects_bad_buffers():
    from openhomelbm_b200 import coupling

    xfrc = torch.zeros((2, 5, 6), device="cuda")
    with pytest.raises(ValueError):
        coupling.fill_xfrc(xfrc, torch.tensor([1], dtype=torch.int64, device="cuda"), torch.zeros((2, 1, 3), device="cuda"),
                           torch.zeros((2, 1, 3), device="cuda"))
    with pytest.raises(ValueError):
        coupling.fill_xfrc(xfrc.cpu(), torch.tensor([1], dtype=torch.int32), torch.zeros((2, 1, 3)), torch.zeros((2, 1, 3)))
    # an out-of-range body id is skipped on the device: nothing else is written
    coupling.fill_xfrc(xfrc, torch.tensor([7], dtype=torch.int32, device="cuda"), torch.ones((2, 1, 3), device="cuda"),
                       torch.ones((2, 1, 3), device="cuda"))
    torch.cuda.synchronize()
    assert float(xfrc.abs().sum()) == 0.0
