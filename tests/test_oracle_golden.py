"""The CPU oracle against the golden fixtures made by running the reference's own kernels.

tests/golden/make_golden.py executes the reference's Warp kernel source (launch order of
Warp's CPU backend, binary32, no FMA) through tests/golden/warp_emu.py. The float build of
the oracle must reproduce every stored step bit for bit, including the per-solid loads
that the reference accumulates with ``wp.atomic_add`` in thread order.
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as orc


def _solids2d(g):
    n = int(g["n_objects"])
    return orc.Solids2D(line=g["solid_line"], line_num=g["solid_line_num"],
                        position=g["solid_position0"].copy(), angle=g["solid_angle0"].copy(),
                        scale=g["solid_scale"], mass_center=g["solid_mass_center"],
                        max_radius=g["solid_max_radius"]).cast(np.float32) if n else None


@pytest.mark.parametrize("case", ["d2q9_walls", "d2q9_bc_types", "d2q9_solids"])
def test_oracle_matches_reference_2d(case):
    g = load_golden(case)
    m = g["init_moments"]
    prev = m.copy()
    s = _solids2d(g)
    vx, vy, om = (np.float32(v) for v in g["motion"])
    for step in range(int(g["steps"])):
        if s is not None and (vx or vy or om):
            # advance_prescribed_solid_motion_kernel, envs/lbm/karman/karman_lbm_env.py:65-77
            s.position[0] = s.position[0] + np.array([vx, vy], np.float32)
            s.angle[0] = s.angle[0] + om
        new, loads = orc.step_2d(m, prev, vis_shear=g["vis_shear"], bc_type=g["bc_type"],
                               bc_value=g["bc_value"], flag=g["flag"], forcex=g["forcex"],
                               forcey=g["forcey"], solids=s, grid_length=g["grid_length"],
                               time_step=g["time_step"])
        m, prev = new, m
        np.testing.assert_array_equal(m, g["moments"][step], err_msg=f"{case} step {step}")
        if s is not None:
            np.testing.assert_array_equal(loads.T, g["solid_loads"][step], err_msg=f"loads step {step}")
            np.testing.assert_array_equal(s.tf, g["solid_line_transformed"][step])
            np.testing.assert_array_equal(s.tf_last, g["solid_line_transformed_last"][step])


def _pose_update(s, pos, q_wxyz, first):
    """convert_and_update_solid_batch_3d, envs/lbm3d/lbm_fluid_env_3d_func.py:42-100,
    with mujoco_origin 0, lbm_origin 0 and scale 1 (the fixture's mapping)."""
    new = np.array([pos[0], pos[1], pos[2], q_wxyz[1], q_wxyz[2], q_wxyz[3], q_wxyz[0]], np.float32)
    if not first:
        s.transforms_last[0] = s.transforms[0]
    s.transforms[0] = new
    if first:
        s.transforms_last[0] = new
        s.initialized[0] = 1
    s.position[0] = pos


@pytest.mark.parametrize("case", ["d3q27_walls", "d3q27_periodic", "d3q27_mesh"])
def test_oracle_matches_reference_3d(case):
    g = load_golden(case)
    periodic = bool(g["periodic"])
    m = g["init_moments"]
    prev = m.copy()
    nx, ny, nz = (int(v) for v in g["shape"])
    flag = None if periodic else orc.border_flags_3d(nx, ny, nz)
    s = None
    if "mesh_vertices" in g:
        tris = g["mesh_vertices"][g["mesh_faces"]]
        s = orc.Solids3D(tri_offset=np.array([0, len(tris)]), tris=tris,
                         transforms=np.zeros((1, 7)), transforms_last=np.zeros((1, 7)),
                         initialized=np.zeros(1), position=np.zeros((1, 3)),
                         bound_radius=g["bound_radius"]).cast(np.float32)
    for step in range(int(g["steps"])):
        if s is not None:
            _pose_update(s, g["poses_pos"][step], g["poses_quat_wxyz"][step], step == 0)
            np.testing.assert_array_equal(np.stack([s.transforms[0], s.transforms_last[0]]),
                                          g["transforms"][step])
        new, loads = orc.step_3d(m, prev, vis_shear=g["vis_shear"], bc_type=g["bc_type"],
                               bc_value=g["bc_value"], flag=flag, force=g["force"], solids=s,
                               periodic=periodic)
        m, prev = new, m
        np.testing.assert_array_equal(m, g["moments"][step], err_msg=f"{case} step {step}")
        if s is not None:
            np.testing.assert_array_equal(loads[0], g["solid_loads"][step], err_msg=f"loads {step}")


def test_oracle_threads_match_single_thread():
    """The threaded oracle (the CPU baseline) computes the same moments as the serial one."""
    g = load_golden("d3q27_periodic")
    a, _ = orc.step_3d(g["init_moments"], vis_shear=g["vis_shear"], periodic=True, nthreads=1)
    b, _ = orc.step_3d(g["init_moments"], vis_shear=g["vis_shear"], periodic=True, nthreads=3)
    np.testing.assert_array_equal(a, b)
