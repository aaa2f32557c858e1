"""D2Q9 CUDA step (stream-collide, polygon cut cells, momentum exchange, apply_bc) against the
reference (golden fixtures) and the oracle.

Moments: the parity criterion of oracle.oracle.check_parity (relative L2 of rho, u, Pi/rho
below 1e-5 against the binary32 reference, and no less accurate than the reference against
the binary64 evaluation of the same algorithm). Per-solid loads: the reference sums
them in binary32 with atomics and the CUDA path in binary64, so they agree to the binary32
summation error, checked at 1e-4 relative to the largest load component.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-5


def make_solver(nx, ny, vis, bc_type, bc_value, init=None, forcex=None, forcey=None, n_objects=1,
                storage="float32"):
    from openhomelbm_b200.lbm import LBM_Solver

    s = LBM_Solver(nx, ny, solid_num=n_objects, use_graph=False, storage=storage)
    f = s.flows[0]
    f.vis_shear = float(vis)
    f.bc_type = list(map(int, bc_type))
    f.bc_value = np.asarray(bc_value, np.float32)
    if init is not None:
        t = torch.tensor(init, device=f.device, dtype=f.moments[0].dtype)
        f.moments[0].copy_(t)
        f.moments[1].copy_(t)
    if forcex is not None:
        f.force[0].copy_(torch.tensor(forcex, device=f.device))
        f.force[1].copy_(torch.tensor(forcey, device=f.device))
        f.use_force = True
    return s


def _configure_from_golden(s, g):
    f = s.flows[0]
    n = int(g["n_objects"])
    for sid in range(n):
        k = int(g["solid_line_num"][sid])
        if k == 0:
            continue
        f.configure_solid(sid, g["solid_line"][sid, :k], tuple(g["solid_position0"][sid]),
                          angle=float(g["solid_angle0"][sid]), scale=float(g["solid_scale"][sid]))
        # the reference computes max_radius in float64 then stores binary32; reuse its value
        f.solid_max_radius[sid] = float(g["solid_max_radius"][sid])


@pytest.mark.parametrize("case", ["d2q9_walls", "d2q9_bc_types", "d2q9_solids"])
def test_d2q9_matches_reference_fixture(case):
    g = load_golden(case)
    nx, ny = int(g["nx"]), int(g["ny"])
    s = make_solver(nx, ny, g["vis_shear"], g["bc_type"], g["bc_value"], init=g["init_moments"],
                    forcex=g["forcex"], forcey=g["forcey"], n_objects=int(g["n_objects"]))
    f = s.flows[0]
    f.flag.copy_(torch.tensor(g["flag"], device=f.device))
    _configure_from_golden(s, g)
    vx, vy, om = (float(v) for v in g["motion"])
    has_solids = int(g["solid_line_num"].max()) > 0
    sol64 = None
    if has_solids:
        sol64 = orc.Solids2D(line=g["solid_line"], line_num=g["solid_line_num"],
                             position=g["solid_position0"].astype(np.float64),
                             angle=g["solid_angle0"].astype(np.float64), scale=g["solid_scale"],
                             mass_center=g["solid_mass_center"], max_radius=g["solid_max_radius"]).cast(np.float64)
    m64 = g["init_moments"].astype(np.float64)
    p64 = m64.copy()
    for step in range(int(g["steps"])):
        if has_solids and (vx or vy or om):
            f.solid_position[0] += torch.tensor([vx, vy], device=f.device)
            f.solid_angle[0] += om
            sol64.position[0] += np.array([np.float32(vx), np.float32(vy)], np.float64)
            sol64.angle[0] += np.float64(np.float32(om))
        s.step()
        new, _ = orc.step_2d(m64, p64, vis_shear=float(g["vis_shear"]), bc_type=g["bc_type"],
                             bc_value=g["bc_value"], flag=g["flag"], forcex=g["forcex"], forcey=g["forcey"],
                             solids=sol64, grid_length=float(g["grid_length"]), dtype=np.float64)
        m64, p64 = new, m64
        msgs = orc.check_parity(f.cur.cpu().numpy(), g["moments"][step], m64)
        assert not msgs, (step, msgs)
        if has_solids:
            torch.cuda.synchronize()
            got = torch.stack([f.solid_forcex, f.solid_forcey, f.torque]).cpu().numpy()
            ref = g["solid_loads"][step]
            scale = np.abs(ref).max()
            assert np.abs(got - ref).max() <= 1e-4 * scale + 1e-7, (step, got, ref)
            np.testing.assert_allclose(f.solid_line_transformed.cpu().numpy(), g["solid_line_transformed"][step],
                                       rtol=0, atol=2e-5)


def test_d2q9_cylinder_wake_100_steps_vs_oracle():
    """A small Karman configuration: inflow left, zero-gradient elsewhere, 96-gon cylinder."""
    nx, ny, vis, u_in = 96, 48, 0.02, 0.05
    circle = np.stack([np.cos(np.linspace(0, 2 * np.pi, 96, endpoint=False)),
                       np.sin(np.linspace(0, 2 * np.pi, 96, endpoint=False))], 1).astype(np.float32)
    bc_type = [0, 1, 1, 1]
    bc_value = [[u_in, 0.0], [0, 0], [0, 0], [0, 0]]
    rng = np.random.default_rng(0)
    m0 = np.zeros((6, nx, ny), np.float32)
    m0[0] = 1.0
    m0[1] = u_in + rng.uniform(-1e-3, 1e-3, (nx, ny))
    m0[2] = rng.uniform(-1e-3, 1e-3, (nx, ny))
    s = make_solver(nx, ny, vis, bc_type, bc_value, init=m0)
    f = s.flows[0]
    f.configure_solid(0, circle, (24.0, 24.3), angle=0.0, scale=6.0 / nx)
    mr = float(f.solid_max_radius[0].item())
    steps = 100
    loads_gpu = []
    for _ in range(steps):
        s.step()
        loads_gpu.append(torch.stack([f.solid_forcex, f.solid_forcey, f.torque]).cpu().numpy())
    sol = orc.Solids2D(line=circle[None], line_num=np.array([96]), position=np.array([[24.0, 24.3]]),
                       angle=np.zeros(1), scale=np.array([6.0 / nx]), mass_center=np.zeros((1, 2)),
                       max_radius=np.array([mr])).cast(np.float32)
    sol64 = orc.Solids2D(line=circle[None], line_num=np.array([96]), position=np.array([[24.0, 24.3]]),
                         angle=np.zeros(1), scale=np.array([np.float32(6.0 / nx)]), mass_center=np.zeros((1, 2)),
                         max_radius=np.array([mr])).cast(np.float64)
    flag = orc.border_flags_2d(nx, ny)
    m, prev = m0.copy(), m0.copy()
    m64, p64 = m0.astype(np.float64), m0.astype(np.float64)
    for k in range(steps):
        new, loads = orc.step_2d(m, prev, vis_shear=np.float32(vis), bc_type=bc_type, bc_value=bc_value,
                                 flag=flag, solids=sol)
        m, prev = new, m
        new, _ = orc.step_2d(m64, p64, vis_shear=float(np.float32(vis)), bc_type=bc_type, bc_value=bc_value,
                             flag=flag, solids=sol64, dtype=np.float64)
        m64, p64 = new, m64
    msgs = orc.check_parity(f.cur.cpu().numpy(), m, m64)
    assert not msgs, msgs
    ref = loads[0]
    got = loads_gpu[-1][:, 0]
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max(), (got, ref)


def test_d2q9_graph_replay_equals_eager():
    nx, ny = 64, 40
    circle = np.stack([np.cos(np.linspace(0, 2 * np.pi, 32, endpoint=False)),
                       np.sin(np.linspace(0, 2 * np.pi, 32, endpoint=False))], 1)
    out = []
    for use_graph in (False, True):
        s = make_solver(nx, ny, 0.02, [0, 1, 1, 1], [[0.05, 0], [0, 0], [0, 0], [0, 0]])
        s.use_graph = use_graph
        s.set_uniform_flow(0.05, 0.0)
        f = s.flows[0]
        f.configure_solid(0, circle, (20.0, 20.0), scale=4.0 / nx)
        for k in range(9):
            f.solid_position[0] += torch.tensor([0.01, 0.005], device=f.device)
            f.bc_value = np.array([[0.05, 0.001 * k], [0, 0], [0, 0], [0, 0]], np.float32)
            s.step()
        out.append((f.cur.clone(), f.torque.clone()))
    assert torch.equal(out[0][0], out[1][0])
    assert torch.allclose(out[0][1], out[1][1], rtol=1e-6, atol=1e-9)


def test_d2q9_uniform_init_matches_reference_fixture():
    """set_uniform_flow_kernel / InitBoundary against the reference's own kernels."""
    from openhomelbm_b200.lbm import LBM_Solver

    g = load_golden("init")
    s = LBM_Solver(7, 5, use_graph=False)
    s.set_uniform_flow(*(float(v) for v in g["u2"]))
    f = s.flows[0]
    np.testing.assert_array_equal(f.flag.cpu().numpy(), g["flag2"])
    # the reference forms S from sums of populations of size ~1/3: two ulps of 1/3
    for buf, ref in ((f.cur, g["moments2"]), (f.post, g["post2"])):
        np.testing.assert_allclose(buf.cpu().numpy(), ref, rtol=0, atol=6e-8)


def test_create_solid_from_mujoco_uses_the_geometry_projection():
    """LBM_Solver.create_solid_from_mujoco on a stand-in MuJoCo model (MuJoCo's field names):
    the solid equals create_solid_from_polygon with the projection of
    openhomelbm_b200.geometry.extract_lbm_polygon_from_mujoco, and the MuJoCo mapping records
    the body's xy position."""
    from test_geometry import _fake_model

    from openhomelbm_b200.geometry import extract_lbm_polygon_from_mujoco
    from openhomelbm_b200.lbm import LBM_Solver

    model, data, _ = _fake_model()
    a = LBM_Solver(64, 48, solid_num=1, use_graph=False)
    info = a.create_solid_from_mujoco(0, model, data, "b", lbm_position=(30.0, 24.0), lbm_scale=0.2)
    ref = extract_lbm_polygon_from_mujoco(model, data, "b")
    np.testing.assert_array_equal(info["vertices"], ref["vertices"])
    b = LBM_Solver(64, 48, solid_num=1, use_graph=False)
    b.create_solid_from_polygon(0, ref["vertices"], (30.0, 24.0), 0.2, ref["angle"], mujoco_origin=ref["position"])
    fa, fb = a.flows[0], b.flows[0]
    for name in ("solid_line", "solid_line_num", "solid_position", "solid_angle", "solid_scale", "solid_max_radius"):
        assert torch.equal(getattr(fa, name), getattr(fb, name)), name
    assert int(fa.solid_line_num[0]) == len(ref["vertices"]) > 3
    np.testing.assert_allclose(a.mujoco_mappings[0]["mujoco_origin"], [3.0, 3.0])
    assert a.mujoco_mappings[0]["scale"] == pytest.approx(0.2 * 64)
