"""Immersed triangle-mesh solids of the D3Q27 step on the GPU: cut links, wall velocity and
momentum exchange (stream_and_collide_3d's narrow band, envs/lbm3d/lbm_func_3d.py:364-604),
against the reference's own run (golden fixture) and the oracle.

Moments use the parity criterion of oracle.check_parity (relative L2 below 1e-5 against the
binary32 reference, max error against binary64 within 3x the reference's own binary32 error).
Loads (force, torque) are sums of a few hundred link terms: the GPU sums them in binary64,
the reference in binary32 atomics, so they are checked against the binary64 oracle with an
error bound of 3x the reference's own binary32 error plus 1e-6 of the load scale.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _loads_ok(got, ref32, ref64):
    got, ref32, ref64 = (np.asarray(a, np.float64) for a in (got, ref32, ref64))
    scale = max(np.abs(ref64).max(), 1e-12)
    return np.abs(got - ref64).max() <= 3 * np.abs(ref32 - ref64).max() + 1e-6 * scale


def _solids_from(s, k=0):
    """The solver's solid state of world k as oracle Solids3D (same transforms and poses)."""
    f = s.flows[k]
    tris = s._tris.cpu().numpy()
    return orc.Solids3D(tri_offset=s._tri_offset.cpu().numpy(), tris=tris,
                        transforms=f.mesh_transforms.cpu().numpy(), transforms_last=f.mesh_transforms_last.cpu().numpy(),
                        initialized=f.mesh_transforms_initialized.cpu().numpy(), position=f.solid_position.cpu().numpy(),
                        bound_radius=f.solid_bound_radius.cpu().numpy(),
                        scale_sizes=f.mesh_scale_sizes.cpu().numpy())


def test_mesh_cut_links_match_reference_fixture():
    """An octahedron moving and turning through a walled 12x11x12 box, 3 steps (the reference's
    kernels run on the same inputs produced the fixture)."""
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    g = load_golden("d3q27_mesh")
    nx, ny, nz = (int(v) for v in g["shape"])
    s = LBM_Solver3D(nx, ny, nz, solid_num=1, use_graph=False)
    f = s.flows[0]
    f.vis_shear = float(g["vis_shear"])
    f.bc_type = list(map(int, g["bc_type"]))
    f.bc_value = np.asarray(g["bc_value"], np.float32)
    t = torch.tensor(g["init_moments"], device=f.device)
    f.moments[0].copy_(t)
    f.moments[1].copy_(t)
    f.force.copy_(torch.tensor(g["force"], device=f.device))
    f.use_force = True
    # vertices are already in lattice units: lbm_scale * nx = 1 exactly
    s.create_solid_from_mesh(0, (g["mesh_vertices"], g["mesh_faces"]), lbm_position=tuple(g["poses_pos"][0]),
                             lbm_scale=1.0 / nx)
    assert np.isclose(float(f.solid_bound_radius[0]), float(g["bound_radius"][0]), rtol=0, atol=0)
    flag = orc.border_flags_3d(nx, ny, nz)
    m64 = g["init_moments"].astype(np.float64)
    p64 = m64.copy()
    for step in range(int(g["steps"])):
        # the pose the reference's coupling kernel produced for this step
        f.solid_position[0] = torch.tensor(g["poses_pos"][step], device=f.device)
        f.mesh_transforms[0] = torch.tensor(g["transforms"][step][0], device=f.device)
        f.mesh_transforms_last[0] = torch.tensor(g["transforms"][step][1], device=f.device)
        f.mesh_transforms_initialized[0] = 1
        solids = _solids_from(s).cast(np.float64)
        s.step()
        new, loads64 = orc.step_3d(m64, p64, vis_shear=float(g["vis_shear"]), bc_type=g["bc_type"],
                                   bc_value=g["bc_value"], flag=flag, force=g["force"], solids=solids,
                                   dtype=np.float64)
        m64, p64 = new, m64
        msgs = orc.check_parity(f.cur.cpu().numpy(), g["moments"][step], m64)
        assert not msgs, (step, msgs)
        got = np.concatenate([f.solid_force[0].cpu().numpy(), f.solid_torque[0].cpu().numpy()])
        assert np.abs(got).max() > 0
        assert _loads_ok(got, g["solid_loads"][step], loads64[0]), (step, got, g["solid_loads"][step], loads64[0])


def _icosahedron():
    from scipy.spatial import ConvexHull

    p = (1 + 5 ** 0.5) / 2
    v = []
    for a in (-1, 1):
        for b in (-p, p):
            v += [(0, a, b), (a, b, 0), (b, 0, a)]
    v = np.array(v, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, ConvexHull(v).simplices.astype(np.int64)


def _quat(axis, angle):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    return np.concatenate([[np.cos(angle / 2)], np.sin(angle / 2) * a]).astype(np.float32)  # w, x, y, z


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_two_moving_meshes_tma_path_vs_oracle(storage):
    """Two icosahedra whose bands overlap, moving and turning in a walled 64x48x64 box (the
    TMA stream-collide kernel plus the band), poses set by the coupling kernel each step and
    the step replayed from a CUDA graph; 8 steps against the oracle."""
    from openhomelbm_b200 import coupling
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    nx, ny, nz = 64, 48, 64
    u = (0.03, -0.01, 0.02)
    kw = dict(storage=storage, u_scale=0.05, s_scale=0.0025) if storage != "float32" else {}
    s = LBM_Solver3D(nx, ny, nz, solid_num=2, **kw)
    f = s.flows[0]
    f.vis_shear = 0.02
    f.bc_type = [0, 1, 1, 1, 1, 1]
    f.bc_value = np.array([u] + [(0, 0, 0)] * 5, np.float32)
    s.set_uniform_flow(*u)
    verts, faces = _icosahedron()
    p0 = [np.array([30.2, 23.6, 31.1]), np.array([38.7, 25.3, 33.4])]
    vel = [np.array([0.04, 0.01, -0.02]), np.array([-0.03, 0.02, 0.01])]
    for k in range(2):
        s.create_solid_from_mesh(k, (verts, faces), lbm_position=tuple(p0[k]), lbm_scale=5.5 / nx,
                                 init_quaternion=tuple(_quat((1, 2, 3), 0.1 * k)))
    ids = torch.tensor([0, 1], dtype=torch.int32, device=f.device)
    zeros = torch.zeros((2, 3), device=f.device)
    ones = torch.ones(2, device=f.device)
    flag = orc.border_flags_3d(nx, ny, nz)
    f32 = lambda a: a.float().cpu().numpy() if a.dtype != torch.float32 else a.cpu().numpy()
    m0 = f.decoded().double().cpu().numpy()
    m32, p32 = m0.astype(np.float32), m0.astype(np.float32)
    m64, p64 = m0.copy(), m0.copy()
    steps = 8
    for step in range(steps):
        pos = np.stack([p0[k] + vel[k] * (step + 1) for k in range(2)]).astype(np.float32)
        quat = np.stack([_quat((1, 2, 3), 0.1 * k + 0.05 * (step + 1)) for k in range(2)])
        coupling.convert_and_update_solid_batch_3d(s, ids, torch.tensor(pos[None], device=f.device),
                                                   torch.tensor(quat[None], device=f.device),
                                                   mujoco_origins=zeros, lbm_origins=zeros, scales=ones)
        solids = _solids_from(s)
        np.testing.assert_array_equal(solids.position, pos)
        s.step()
        new, l32 = orc.step_3d(m32, p32, vis_shear=np.float32(0.02), bc_type=f.bc_type, bc_value=f.bc_value,
                               flag=flag, solids=solids.cast(np.float32), nthreads=0)
        m32, p32 = new, m32
        new, l64 = orc.step_3d(m64, p64, vis_shear=float(np.float32(0.02)), bc_type=f.bc_type, bc_value=f.bc_value,
                               flag=flag, solids=_solids_from(s).cast(np.float64), dtype=np.float64, nthreads=0)
        m64, p64 = new, m64
        got = np.concatenate([f32(f.solid_force), f32(f.solid_torque)], axis=1)
        assert np.abs(got).max() > 0
        if storage == "float32":
            assert _loads_ok(got, l32, l64), (step, got, l32, l64)
    got = f.decoded().double().cpu().numpy()
    if storage == "float32":
        msgs = orc.check_parity(got, m32, m64)
        assert not msgs, msgs
    else:
        # reduced storage: velocity L2 against binary64 within the float16 bound of the plain tests
        err = np.linalg.norm(got[1:4] - m64[1:4]) / np.linalg.norm(m64[1:4])
        assert err < 1e-3, err
        assert np.abs(got[0] - m64[0]).max() < 5e-3


def test_solid_links_rejects_bad_arguments():
    import ctypes

    from openhomelbm_b200 import _lib
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    s = LBM_Solver3D(16, 16, 32, solid_num=2, use_graph=False)
    s.create_solid_from_mesh(0, _icosahedron(), lbm_position=(8, 8, 16), lbm_scale=0.2)
    w = s.flows[0].world_struct()
    st = s._solids_struct(0)
    st.n_objects = 65
    rc = _lib.lib().hl_d3q27_solid_links(ctypes.byref(w), 0.02, ctypes.byref(st), _lib.stream_ptr())
    assert rc == _lib.HL_ERR_ARG
    with pytest.raises(ValueError):
        s.create_solid_from_mesh(2, _icosahedron())


def test_mjcf_body_mesh_vs_oracle(tmp_path):
    """A body meshed from MJCF by openhomelbm_b200.geometry (a capsule given by fromto and a
    box, merged into one closed triangle mesh) as the solid of a walled 48x40x40 box: 4 steps
    against the oracle, binary32 storage."""
    from openhomelbm_b200 import geometry
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    p = tmp_path / "fish.xml"
    p.write_text('<mujoco model="fish"><worldbody><body name="torso" pos="0 0 0">'
                 '<geom type="capsule" fromto="-0.3 0 0 0.3 0 0" size="0.12"/>'
                 '<geom type="box" size="0.1 0.05 0.2" pos="0.3 0 0"/></body></worldbody></mujoco>')
    mesh = geometry.parse_mjcf_to_meshes(str(p))["torso"]
    nx, ny, nz = 48, 40, 40
    u = (0.03, 0.0, 0.01)
    s = LBM_Solver3D(nx, ny, nz, solid_num=1)
    f = s.flows[0]
    f.vis_shear = 0.02
    f.bc_type = [0, 1, 1, 1, 1, 1]
    f.bc_value = np.array([u] + [(0, 0, 0)] * 5, np.float32)
    s.set_uniform_flow(*u)
    s.create_solid_from_mesh(0, mesh, lbm_position=(20.3, 19.6, 20.4), lbm_scale=20.0 / nx,
                                    init_quaternion=tuple(_quat((0, 1, 1), 0.4)))
    assert abs(float(f.solid_bound_radius[0]) - 9.0) < 1e-4  # box corner (0.4, 0.05, 0.2) x 20
    flag = orc.border_flags_3d(nx, ny, nz)
    m0 = f.decoded().double().cpu().numpy()
    m32, p32 = m0.astype(np.float32), m0.astype(np.float32)
    m64, p64 = m0.copy(), m0.copy()
    for step in range(4):
        solids = _solids_from(s)
        s.step()
        new, l32 = orc.step_3d(m32, p32, vis_shear=np.float32(0.02), bc_type=f.bc_type, bc_value=f.bc_value,
                               flag=flag, solids=solids.cast(np.float32), nthreads=0)
        m32, p32 = new, m32
        new, l64 = orc.step_3d(m64, p64, vis_shear=float(np.float32(0.02)), bc_type=f.bc_type, bc_value=f.bc_value,
                               flag=flag, solids=_solids_from(s).cast(np.float64), dtype=np.float64, nthreads=0)
        m64, p64 = new, m64
        got = np.concatenate([f.solid_force.cpu().numpy(), f.solid_torque.cpu().numpy()], axis=1)
        assert np.abs(got).max() > 0
        assert _loads_ok(got, l32, l64), (step, got, l32, l64)
    msgs = orc.check_parity(f.decoded().double().cpu().numpy(), m32, m64)
    assert not msgs, msgs


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_band_form_equals_work_list_form(storage):
    """hl_d3q27_solid_links with and without the work list (a block row per solid over its
    band box, or the listed cells taken in turn by a fixed grid) computes the same cells with
    the same code: identical moments; loads equal up to the order of their binary64 sums.
    A served swimmer (5 ellipsoid segments, 1800 triangles) in a 96^3 box after 3 steps."""
    from openhomelbm_b200 import _lib, serving

    r = serving.Request(0, 96, 4321, 0.0, control_steps=4)
    d = serving.Domain(r, storage, 0.01, torch.device("cuda:0"), use_graph=False)
    for step in range(3):
        d.stage_poses(step)
        d.launch()
        d.event.synchronize()
    s = d.solver
    f = s.flows[0]
    st = _lib.stream_ptr()
    out = []
    for work_list in (True, False):
        s.use_work_list = work_list
        f.moments[f.parity ^ 1].zero_()
        s._launch(f.parity, st)
        torch.cuda.synchronize()
        out.append((f.moments[f.parity ^ 1].clone(), f.solid_force.clone(), f.solid_torque.clone()))
    s.use_work_list = True
    assert torch.equal(out[0][0], out[1][0])
    for k in (1, 2):
        a, b = out[0][k].double(), out[1][k].double()
        assert a.abs().max() > 0
        assert torch.allclose(a, b, rtol=1e-6, atol=1e-6 * float(a.abs().max()))
