"""Generate the golden fixtures in this folder by running the reference's own kernels.

The reference (kuiwuchn/OpenHOMELBM) is Python whose GPU work is NVIDIA Warp kernels. Warp
is not installable here, so this script installs ``warp_emu`` (a CPU emulation of the Warp
builtins those kernels call) as the ``warp`` module, imports the reference's kernel modules
from their source tree, and launches the kernels in the order the reference's solvers
launch them:

* 2D, ``LBM_Solver.step`` (envs/lbm/lbm_solver.py:104-141): zero the per-solid loads,
  ``precompute_transformed_segments`` -> ``stream_and_collide`` -> ``apply_bc`` ->
  ``Swap_Mom``; prescribed solid motion through ``advance_prescribed_solid_motion_kernel``
  (envs/lbm/karman/karman_lbm_env.py:65-77) before each step.
* 3D, ``LBM_Solver3D.step`` (envs/lbm3d/lbm_solver_3d.py:95-127): ``init_force_3d_batch``
  -> ``stream_and_collide_3d`` -> ``apply_bc_3d`` -> ``Swap_Mom_3D``; poses enter through
  ``convert_and_update_solid_batch_3d`` (envs/lbm3d/lbm_fluid_env_3d_func.py:42-100).
* 3D periodic: the reference has no periodic boundary, so the periodic case runs the
  reference kernel on an (n+2)^3 grid whose ghost shell is WALL and is refilled with the
  periodic images of the interior after every ``stream_and_collide_3d`` (no ``apply_bc_3d``).

Usage (needs the reference source tree; the fixtures it writes are committed):

    python tests/golden/make_golden.py --reference <reference source tree>

(or the HOMELBM_REFERENCE environment variable instead of --reference)
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import warp_emu  # noqa: E402


def import_reference(ref):
    wp = warp_emu.install()

    def pkg(name, path):
        m = types.ModuleType(name)
        m.__path__ = [path]
        sys.modules[name] = m
        return m

    pkg("refenvs", f"{ref}/envs")
    pkg("refenvs.lbm", f"{ref}/envs/lbm")
    pkg("refenvs.lbm3d", f"{ref}/envs/lbm3d")
    pkg("refenvs.lbm.karman", f"{ref}/envs/lbm/karman")
    pkg("refenvs.lbm3d.karman", f"{ref}/envs/lbm3d/karman")
    stub3 = types.ModuleType("refenvs.lbm3d.lbm_fluid_env_3d")
    stub3.LBMFluidEnv3D = object
    sys.modules["refenvs.lbm3d.lbm_fluid_env_3d"] = stub3
    # the gym environment base class is not needed by the kernels; stand it in
    stub = types.ModuleType("refenvs.lbm.lbm_fluid_env")
    stub.LBMFluidEnv = object
    sys.modules["refenvs.lbm.lbm_fluid_env"] = stub
    mods = types.SimpleNamespace(wp=wp, root=ref)
    mods.core2 = importlib.import_module("refenvs.lbm.lbm_core")
    mods.func2 = importlib.import_module("refenvs.lbm.lbm_func")
    mods.solid = importlib.import_module("refenvs.lbm.solid_func")
    mods.karman2 = importlib.import_module("refenvs.lbm.karman.karman_lbm_env")
    mods.couple2 = importlib.import_module("refenvs.lbm.lbm_fluid_env_func")
    mods.core3 = importlib.import_module("refenvs.lbm3d.lbm_core_3d")
    mods.func3 = importlib.import_module("refenvs.lbm3d.lbm_func_3d")
    mods.couple3 = importlib.import_module("refenvs.lbm3d.lbm_fluid_env_3d_func")
    mods.karman3 = importlib.import_module("refenvs.lbm3d.karman.karman_lbm_env_3d")
    return mods


# --------------------------------------------------------------------------- 2D
def _moments2d(flow):
    return np.stack([flow.rho.np, flow.u.np[..., 0], flow.u.np[..., 1],
                     flow.Sxx.np, flow.Syy.np, flow.Sxy.np]).astype(np.float32)


def _set_moments2d(flow, m):
    flow.rho.np[...] = m[0]
    flow.u.np[..., 0] = m[1]
    flow.u.np[..., 1] = m[2]
    flow.Sxx.np[...] = m[3]
    flow.Syy.np[...] = m[4]
    flow.Sxy.np[...] = m[5]
    flow.rho_post.np[...] = m[0]
    flow.u_post.np[..., 0] = m[1]
    flow.u_post.np[..., 1] = m[2]
    flow.Sxx_post.np[...] = m[3]
    flow.Syy_post.np[...] = m[4]
    flow.Sxy_post.np[...] = m[5]


def case_2d(R, name, nx, ny, steps, seed, vis, bc_type, bc_value, solids, motion, init,
            force_amp):
    wp = R.wp
    rng = np.random.default_rng(seed)
    flow = R.core2.HomeFlow()
    flow.Initialize(nx, ny, n_objects=max(1, len(solids)))
    flow.vis_shear = vis
    flow.bc_type = wp.types.vector(length=4, dtype=wp.int32)(*bc_type)
    flow.bc_value = wp.array(tuple(wp.vec2(*v) for v in bc_value), dtype=wp.vec2)
    for sid, s in enumerate(solids):
        flow.configure_solid(sid, np.asarray(s["lines"], np.float32), tuple(s["position"]),
                             angle=s["angle"], scale=s["scale"])
    flows = wp.array([flow], dtype=R.core2.HomeFlow)
    wp.launch(R.func2.InitBoundary, dim=(1, nx, ny), inputs=[flows])
    if init == "uniform":
        ux, uy = bc_value[0]
        wp.launch(R.karman2.set_uniform_flow_kernel, dim=(1, nx, ny), inputs=[flows, ux, uy])
        noise = rng.uniform(-1e-3, 1e-3, size=(nx, ny, 2)).astype(np.float32)
        flow.u.np[...] += noise
        flow.u_post.np[...] = flow.u.np
    else:
        wp.launch(R.func2.InitFlow, dim=(1, nx, ny), inputs=[flows])
        m = np.empty((6, nx, ny), np.float32)
        m[0] = 1.0 + rng.uniform(-0.01, 0.01, (nx, ny))
        m[1] = rng.uniform(-0.04, 0.04, (nx, ny))
        m[2] = rng.uniform(-0.04, 0.04, (nx, ny))
        m[3] = m[1] * m[1] + rng.uniform(-2e-3, 2e-3, (nx, ny))
        m[4] = m[2] * m[2] + rng.uniform(-2e-3, 2e-3, (nx, ny))
        m[5] = m[1] * m[2] + rng.uniform(-2e-3, 2e-3, (nx, ny))
        _set_moments2d(flow, m.astype(np.float32))
    if force_amp:
        flow.forcex.np[...] = rng.uniform(-force_amp, force_amp, (nx, ny)).astype(np.float32)
        flow.forcey.np[...] = rng.uniform(-force_amp, force_amp, (nx, ny)).astype(np.float32)

    out = {
        "nx": nx, "ny": ny, "vis_shear": np.float32(vis), "steps": steps,
        "bc_type": np.array(bc_type, np.int32), "bc_value": np.array(bc_value, np.float32),
        "init_moments": _moments2d(flow), "flag": flow.flag.np.copy(),
        "forcex": flow.forcex.np.copy(), "forcey": flow.forcey.np.copy(),
        "n_objects": flow.n_objects, "max_segments": flow.max_segments_per_object,
        "solid_line": flow.solid_line.np.copy(), "solid_line_num": flow.solid_line_num.np.copy(),
        "solid_position0": flow.solid_position.np.copy(), "solid_angle0": flow.solid_angle.np.copy(),
        "solid_scale": flow.solid_scale.np.copy(), "solid_mass_center": flow.solid_mass_center.np.copy(),
        "solid_max_radius": flow.solid_max_radius.np.copy(),
        "motion": np.array(motion if motion else [0.0, 0.0, 0.0], np.float32),
        "grid_length": np.float32(flow.grid_length), "time_step": np.float32(flow.time_step),
    }
    moments, forces, tfs, tfls = [], [], [], []
    for step in range(steps):
        if motion:
            wp.launch(R.karman2.advance_prescribed_solid_motion_kernel, dim=1,
                      inputs=[flows, 0, motion[0], motion[1], motion[2]])
        R.func2.init_force(flow)
        wp.launch(R.func2.precompute_transformed_segments,
                  dim=(1, flow.n_objects, flow.max_segments_per_object), inputs=[flows])
        wp.launch(R.func2.stream_and_collide, dim=(1, nx, ny), inputs=[flows])
        wp.launch(R.func2.apply_bc, dim=(1, nx, ny), inputs=[flows])
        wp.launch(R.func2.Swap_Mom, dim=(1,), inputs=[flows])
        moments.append(_moments2d(flow))
        forces.append(np.stack([flow.solid_forcex.np, flow.solid_forcey.np, flow.torque.np]).copy())
        tfs.append(flow.solid_line_transformed.np.copy())
        tfls.append(flow.solid_line_transformed_last.np.copy())
    out["moments"] = np.stack(moments)
    out["solid_loads"] = np.stack(forces)
    out["solid_line_transformed"] = np.stack(tfs)
    out["solid_line_transformed_last"] = np.stack(tfls)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: {steps} steps, moments finite={np.isfinite(out['moments']).all()}, "
          f"loads={out['solid_loads'][-1].ravel()[:3]}")


# --------------------------------------------------------------------------- 3D
_FIELDS3 = ["rho", "ux", "uy", "uz", "Sxx", "Syy", "Szz", "Sxy", "Sxz", "Syz"]


def _moments3d(flow, post=False):
    sfx = "_post" if post else ""
    u = getattr(flow, "u" + sfx).np
    return np.stack([getattr(flow, "rho" + sfx).np, u[..., 0], u[..., 1], u[..., 2]] +
                    [getattr(flow, n + sfx).np for n in ("Sxx", "Syy", "Szz", "Sxy", "Sxz", "Syz")]
                    ).astype(np.float32)


def _set_moments3d(flow, m):
    for sfx in ("", "_post"):
        getattr(flow, "rho" + sfx).np[...] = m[0]
        u = getattr(flow, "u" + sfx).np
        u[..., 0], u[..., 1], u[..., 2] = m[1], m[2], m[3]
        for k, n in enumerate(("Sxx", "Syy", "Szz", "Sxy", "Sxz", "Syz")):
            getattr(flow, n + sfx).np[...] = m[4 + k]


def _random_moments3d(rng, shape):
    m = np.empty((10,) + shape, np.float32)
    m[0] = 1.0 + rng.uniform(-0.01, 0.01, shape)
    for k in range(3):
        m[1 + k] = rng.uniform(-0.04, 0.04, shape)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    for k, (a, b) in enumerate(pairs):
        m[4 + k] = m[1 + a] * m[1 + b] + rng.uniform(-2e-3, 2e-3, shape)
    return m.astype(np.float32)


def _octahedron(radius):
    v = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]],
                 np.float32) * radius
    f = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4],
                  [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]], np.int32)
    return v, f


def _quat_wxyz(axis, angle):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    h = 0.5 * angle
    return np.array([np.cos(h), *(np.sin(h) * axis)], np.float32)


def case_3d(R, name, shape, steps, seed, vis, bc_type, bc_value, periodic=False,
            mesh=None, force_amp=0.0):
    wp = R.wp
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    gx, gy, gz = (nx + 2, ny + 2, nz + 2) if periodic else (nx, ny, nz)
    n_obj = 1
    flow = R.core3.HomeFlow3D()
    flow.Initialize(gx, gy, gz, n_objects=n_obj)
    flow.vis_shear = vis
    flow.bc_type = wp.types.vector(length=6, dtype=wp.int32)(*bc_type)
    flow.bc_value = wp.array(tuple(wp.vec3(*v) for v in bc_value), dtype=wp.vec3)
    flows = wp.array([flow], dtype=R.core3.HomeFlow3D)
    wp.launch(R.func3.InitBoundary3D, dim=(1, gx, gy, gz), inputs=[flows])
    wp.launch(R.func3.InitFlow3D, dim=(1, gx, gy, gz), inputs=[flows])
    m = _random_moments3d(rng, (nx, ny, nz))
    if periodic:
        full = np.pad(m, ((0, 0), (1, 1), (1, 1), (1, 1)), mode="wrap")
        _set_moments3d(flow, full)
    else:
        _set_moments3d(flow, m)
    if force_amp:
        for c in ("forcex", "forcey", "forcez"):
            f = rng.uniform(-force_amp, force_amp, (nx, ny, nz)).astype(np.float32)
            getattr(flow, c).np[...] = np.pad(f, 1, mode="wrap") if periodic else f

    mesh_info = None
    poses = []
    if mesh is not None:
        verts, faces = _octahedron(mesh["radius"])
        m_wp = wp.Mesh(points=wp.array(verts, dtype=wp.vec3), indices=wp.array(faces.ravel(), dtype=wp.int32))
        flow.mesh_ids.np[0] = m_wp.id
        flow.mesh_scale_sizes.np[0] = (1.0, 1.0, 1.0)
        flow.solid_bound_radius.np[0] = float(np.linalg.norm(verts, axis=1).max())
        mesh_info = (verts, faces)
        for s in range(steps):
            pos = np.asarray(mesh["position"], np.float32) + np.asarray(mesh["velocity"], np.float32) * s
            q = _quat_wxyz(mesh["axis"], mesh["omega"] * s)
            poses.append((pos.astype(np.float32), q))

    out = {"shape": np.array(shape, np.int32), "periodic": int(periodic), "steps": steps,
           "vis_shear": np.float32(vis), "bc_type": np.array(bc_type, np.int32),
           "bc_value": np.array(bc_value, np.float32), "init_moments": m,
           "force": (np.stack([flow.forcex.np, flow.forcey.np, flow.forcez.np])[:, 1:-1, 1:-1, 1:-1]
                     if periodic else np.stack([flow.forcex.np, flow.forcey.np, flow.forcez.np])).copy()}
    if mesh_info is not None:
        out["mesh_vertices"], out["mesh_faces"] = mesh_info
        out["bound_radius"] = flow.solid_bound_radius.np.copy()
        out["poses_pos"] = np.stack([p for p, _ in poses])
        out["poses_quat_wxyz"] = np.stack([q for _, q in poses])
    moments, loads, tfs = [], [], []
    solid_ids = wp.array(np.array([0], np.int32), dtype=wp.int32)
    ones = wp.array(np.array([1.0], np.float32), dtype=wp.float32)
    zero3 = wp.array(np.zeros((1, 3), np.float32), dtype=wp.vec3)
    for step in range(steps):
        if mesh is not None:
            pos, q = poses[step]
            mj_pos = wp.array(pos.reshape(1, 1, 3), dtype=wp.float32)
            mj_quat = wp.array(q.reshape(1, 1, 4), dtype=wp.float32)
            wp.launch(R.couple3.convert_and_update_solid_batch_3d, dim=(1, 1),
                      inputs=[flows, solid_ids, mj_pos, mj_quat, zero3, zero3, ones])
            tfs.append(np.stack([flow.mesh_transforms.np[0], flow.mesh_transforms_last.np[0]]).copy())
        wp.launch(R.func3.init_force_3d_batch, dim=(1,), inputs=[flows])
        wp.launch(R.func3.stream_and_collide_3d, dim=(1, gx, gy, gz), inputs=[flows])
        if periodic:
            post = _moments3d(flow, post=True)
            interior = post[:, 1:-1, 1:-1, 1:-1]
            _set_post3d(flow, np.pad(interior, ((0, 0), (1, 1), (1, 1), (1, 1)), mode="wrap"))
        else:
            wp.launch(R.func3.apply_bc_3d, dim=(1, gx, gy, gz), inputs=[flows])
        wp.launch(R.func3.Swap_Mom_3D, dim=(1,), inputs=[flows])
        cur = _moments3d(flow)
        moments.append(cur[:, 1:-1, 1:-1, 1:-1] if periodic else cur)
        loads.append(np.concatenate([flow.solid_force.np[0], flow.solid_torque.np[0]]).copy())
    out["moments"] = np.stack(moments)
    out["solid_loads"] = np.stack(loads)
    if tfs:
        out["transforms"] = np.stack(tfs)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: {steps} steps, finite={np.isfinite(out['moments']).all()}, loads={out['solid_loads'][-1]}")


def _set_post3d(flow, m):
    flow.rho_post.np[...] = m[0]
    u = flow.u_post.np
    u[..., 0], u[..., 1], u[..., 2] = m[1], m[2], m[3]
    for k, n in enumerate(("Sxx", "Syy", "Szz", "Sxy", "Sxz", "Syz")):
        getattr(flow, n + "_post").np[...] = m[4 + k]


# --------------------------------------------------------------------------- coupling
def case_coupling(R, name, seed):
    """Pose-in and load-out kernels of both coupled environments on random buffers."""
    wp = R.wp
    rng = np.random.default_rng(seed)
    nworld, nbody, nsol = 2, 5, 3
    body_ids = np.array([1, 3, 4], np.int32)
    xipos = rng.uniform(-1, 1, (nworld, nbody, 3)).astype(np.float32)
    q = rng.normal(size=(nworld, nbody, 4))
    xquat = (q / np.linalg.norm(q, axis=-1, keepdims=True)).astype(np.float32)
    mj_origin = rng.uniform(-0.5, 0.5, (nsol, 3)).astype(np.float32)
    lbm_origin = rng.uniform(10, 20, (nsol, 3)).astype(np.float32)
    scales = rng.uniform(20, 40, (nsol,)).astype(np.float32)

    pos_out = wp.zeros((nworld, nsol, 3), dtype=wp.float32)
    quat_out = wp.zeros((nworld, nsol, 4), dtype=wp.float32)
    wp.launch(R.couple3.extract_body_states_3d, dim=(nworld, nsol),
              inputs=[wp.array(xipos, dtype=wp.vec3), wp.array(xquat, dtype=wp.quat),
                      wp.array(body_ids, dtype=wp.int32), pos_out, quat_out])

    flows3 = []
    for _ in range(nworld):
        f = R.core3.HomeFlow3D()
        f.Initialize(6, 6, 6, n_objects=nsol)
        f.solid_force.np[...] = rng.uniform(-1, 1, (nsol, 3))
        f.solid_torque.np[...] = rng.uniform(-1, 1, (nsol, 3))
        flows3.append(f)
    fw3 = wp.array(flows3, dtype=R.core3.HomeFlow3D)
    sids = wp.array(np.arange(nsol, dtype=np.int32), dtype=wp.int32)
    tf_hist = []
    for _ in range(2):  # first call initialises, second moves current -> last
        wp.launch(R.couple3.convert_and_update_solid_batch_3d, dim=(nworld, nsol),
                  inputs=[fw3, sids, pos_out, quat_out, wp.array(mj_origin, dtype=wp.vec3),
                          wp.array(lbm_origin, dtype=wp.vec3), wp.array(scales, dtype=wp.float32)])
        tf_hist.append(np.stack([np.stack([f.mesh_transforms.np, f.mesh_transforms_last.np])
                                 for f in flows3]))
        pos_out.np[...] += np.float32(0.01)
    fo = wp.zeros((nworld, nsol, 3), dtype=wp.float32)
    to = wp.zeros((nworld, nsol, 3), dtype=wp.float32)
    wp.launch(R.couple3.extract_forces_torques_physical_3d, dim=(nworld, nsol),
              inputs=[fw3, sids, 1.7, 0.3, fo, to])
    xfrc = wp.zeros((nworld, nbody), dtype=wp.spatial_vector)
    wp.launch(R.couple3.fill_xfrc_3d_kernel, dim=(nworld, nsol),
              inputs=[xfrc, wp.array(body_ids, dtype=wp.int32), fo, to])

    flows2 = []
    for _ in range(nworld):
        f = R.core2.HomeFlow()
        f.Initialize(6, 6, n_objects=nsol)
        f.solid_forcex.np[...] = rng.uniform(-1, 1, nsol)
        f.solid_forcey.np[...] = rng.uniform(-1, 1, nsol)
        f.torque.np[...] = rng.uniform(-1, 1, nsol)
        flows2.append(f)
    fw2 = wp.array(flows2, dtype=R.core2.HomeFlow)
    wp.launch(R.couple2.convert_and_update_solid_batch_2d, dim=(nworld, nsol),
              inputs=[fw2, sids, pos_out, quat_out, wp.array(mj_origin[:, :2], dtype=wp.float32),
                      wp.array(lbm_origin[:, :2], dtype=wp.float32), wp.array(scales, dtype=wp.float32)])
    fo2 = wp.zeros((nworld, nsol, 3), dtype=wp.float32)
    to2 = wp.zeros((nworld, nsol, 3), dtype=wp.float32)
    wp.launch(R.couple2.extract_forces_torques_batch, dim=(nworld, nsol),
              inputs=[fw2, sids, wp.array(scales, dtype=wp.float32), fo2, to2])
    xfrc2 = wp.zeros((nworld, nbody), dtype=wp.spatial_vector)
    wp.launch(R.couple2.fill_xfrc_kernel, dim=(nworld, nsol),
              inputs=[xfrc2, wp.array(body_ids, dtype=wp.int32), fo2, to2])

    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        body_ids=body_ids, xipos=xipos, xquat=xquat, mj_origin=mj_origin, lbm_origin=lbm_origin,
        scales=scales, pos_out=pos_out.np, quat_out=quat_out.np,
        tf_hist=np.stack(tf_hist), pos_after=pos_out.np.copy(),
        solid_force3=np.stack([f.solid_force.np for f in flows3]),
        solid_torque3=np.stack([f.solid_torque.np for f in flows3]),
        force_conv=np.float32(1.7), torque_conv=np.float32(0.3),
        forces3=fo.np, torques3=to.np, xfrc3=xfrc.np,
        solid_position2=np.stack([f.solid_position.np for f in flows2]),
        solid_angle2=np.stack([f.solid_angle.np for f in flows2]),
        loads2=np.stack([np.stack([f.solid_forcex.np, f.solid_forcey.np, f.torque.np]) for f in flows2]),
        forces2=fo2.np, torques2=to2.np, xfrc2=xfrc2.np)
    print(f"{name}: ok")


def case_init(R, name):
    """The initial-state kernels: InitFlow(3D), set_uniform_flow(_3d)_kernel, InitBoundary."""
    wp = R.wp
    f2 = R.core2.HomeFlow()
    f2.Initialize(7, 5, n_objects=1)
    fw2 = wp.array([f2], dtype=R.core2.HomeFlow)
    wp.launch(R.func2.InitBoundary, dim=(1, 7, 5), inputs=[fw2])
    wp.launch(R.karman2.set_uniform_flow_kernel, dim=(1, 7, 5), inputs=[fw2, 0.07, -0.03])
    f3 = R.core3.HomeFlow3D()
    f3.Initialize(5, 4, 6, n_objects=1)
    fw3 = wp.array([f3], dtype=R.core3.HomeFlow3D)
    wp.launch(R.func3.InitBoundary3D, dim=(1, 5, 4, 6), inputs=[fw3])
    wp.launch(R.karman3.set_uniform_flow_3d_kernel, dim=(1, 5, 4, 6), inputs=[fw3, 0.05, -0.02, 0.03])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                        u2=np.array([0.07, -0.03], np.float32), moments2=_moments2d(f2),
                        post2=np.stack([f2.rho_post.np, f2.u_post.np[..., 0], f2.u_post.np[..., 1],
                                        f2.Sxx_post.np, f2.Syy_post.np, f2.Sxy_post.np]), flag2=f2.flag.np.copy(),
                        u3=np.array([0.05, -0.02, 0.03], np.float32), moments3=_moments3d(f3),
                        post3=_moments3d(f3, post=True), flag3=f3.flag.np.copy())
    print(f"{name}: ok")


def case_reset(R, name, seed):
    """The masked world resets of partial_reset (envs/lbm3d/lbm_fluid_env_3d.py:558-619,
    envs/lbm/lbm_fluid_env.py:305-372): ResetSingleWorldFlow(3D), ResetSingleWorldSolidTransform(3D)
    and ResetSingleWorldForces(3D) over three worlds with random state, mask (1, 0, 1) in 3D and
    (0, 1, 1) in 2D."""
    wp = R.wp
    rng = np.random.default_rng(seed)
    nworld, nsol = 3, 2
    shape3 = (5, 4, 6)
    flows3 = []
    for _ in range(nworld):
        f = R.core3.HomeFlow3D()
        f.Initialize(*shape3, n_objects=nsol)
        _set_moments3d(f, _random_moments3d(rng, shape3))
        _set_post3d(f, _random_moments3d(rng, shape3))
        for n in ("forcex", "forcey", "forcez"):
            getattr(f, n).np[...] = rng.uniform(-1e-3, 1e-3, shape3)
        f.mesh_transforms.np[...] = rng.uniform(-2, 2, f.mesh_transforms.np.shape)
        f.mesh_transforms_last.np[...] = rng.uniform(-2, 2, f.mesh_transforms_last.np.shape)
        f.mesh_transforms_initialized.np[...] = 1
        f.solid_force.np[...] = rng.uniform(-1, 1, (nsol, 3))
        f.solid_torque.np[...] = rng.uniform(-1, 1, (nsol, 3))
        flows3.append(f)

    def snap3(fl):
        return dict(cur=np.stack([_moments3d(f) for f in fl]), post=np.stack([_moments3d(f, post=True) for f in fl]),
                    force=np.stack([np.stack([f.forcex.np, f.forcey.np, f.forcez.np]) for f in fl]),
                    tf=np.stack([f.mesh_transforms.np for f in fl]).astype(np.float32),
                    tf_last=np.stack([f.mesh_transforms_last.np for f in fl]).astype(np.float32),
                    initialized=np.stack([f.mesh_transforms_initialized.np for f in fl]).astype(np.int32),
                    solid_force=np.stack([f.solid_force.np for f in fl]),
                    solid_torque=np.stack([f.solid_torque.np for f in fl]))

    before3 = {k + "3_before": v.copy() for k, v in snap3(flows3).items()}
    fw3 = wp.array(flows3, dtype=R.core3.HomeFlow3D)
    mask3 = np.array([1, 0, 1], np.int32)
    m3 = wp.array(mask3, dtype=wp.int32)
    wp.launch(R.func3.ResetSingleWorldFlow3D, dim=(nworld,) + shape3, inputs=[fw3, m3])
    wp.launch(R.func3.ResetSingleWorldSolidTransform3D, dim=(nworld, nsol, 1), inputs=[fw3, m3])
    wp.launch(R.func3.ResetSingleWorldForces3D, dim=nworld, inputs=[fw3, m3])
    after3 = {k + "3_after": v for k, v in snap3(flows3).items()}

    nx, ny = 7, 5
    square = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float32)
    circle = np.asarray(R.solid.generate_unit_circle_points(6), np.float32)
    flows2 = []
    for _ in range(nworld):
        f = R.core2.HomeFlow()
        f.Initialize(nx, ny, n_objects=nsol)
        f.configure_solid(0, square, (2.5, 2.0), angle=0.1, scale=1.0 / nx)
        f.configure_solid(1, circle, (4.5, 2.5), angle=0.0, scale=0.8 / nx)
        m = np.empty((6, nx, ny), np.float32)
        m[0] = 1.0 + rng.uniform(-0.01, 0.01, (nx, ny))
        m[1:] = rng.uniform(-0.03, 0.03, (5, nx, ny))
        _set_moments2d(f, m)
        f.forcex.np[...] = rng.uniform(-1e-3, 1e-3, (nx, ny))
        f.forcey.np[...] = rng.uniform(-1e-3, 1e-3, (nx, ny))
        f.solid_line_transformed.np[...] = rng.uniform(0, 7, f.solid_line_transformed.np.shape)
        f.solid_line_transformed_last.np[...] = rng.uniform(0, 7, f.solid_line_transformed_last.np.shape)
        f.solid_forcex.np[...] = rng.uniform(-1, 1, nsol)
        f.solid_forcey.np[...] = rng.uniform(-1, 1, nsol)
        f.torque.np[...] = rng.uniform(-1, 1, nsol)
        flows2.append(f)

    def snap2(fl):
        return dict(cur=np.stack([_moments2d(f) for f in fl]),
                    post=np.stack([np.stack([f.rho_post.np, f.u_post.np[..., 0], f.u_post.np[..., 1], f.Sxx_post.np,
                                             f.Syy_post.np, f.Sxy_post.np]) for f in fl]).astype(np.float32),
                    force=np.stack([np.stack([f.forcex.np, f.forcey.np]) for f in fl]),
                    line_tf=np.stack([f.solid_line_transformed.np for f in fl]).astype(np.float32),
                    line_tf_last=np.stack([f.solid_line_transformed_last.np for f in fl]).astype(np.float32),
                    loads=np.stack([np.stack([f.solid_forcex.np, f.solid_forcey.np, f.torque.np]) for f in fl]))

    before2 = {k + "2_before": v.copy() for k, v in snap2(flows2).items()}
    fw2 = wp.array(flows2, dtype=R.core2.HomeFlow)
    mask2 = np.array([0, 1, 1], np.int32)
    m2 = wp.array(mask2, dtype=wp.int32)
    max_seg = flows2[0].max_segments_per_object
    wp.launch(R.func2.ResetSingleWorldFlow, dim=(nworld, nx, ny), inputs=[fw2, m2])
    wp.launch(R.func2.ResetSingleWorldSolidTransform, dim=(nworld, nsol, max_seg), inputs=[fw2, m2])
    wp.launch(R.func2.ResetSingleWorldForces, dim=nworld, inputs=[fw2, m2])
    after2 = {k + "2_after": v for k, v in snap2(flows2).items()}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), mask3=mask3, mask2=mask2,
                        solid_line=np.stack([f.solid_line.np for f in flows2[:1]])[0].astype(np.float32),
                        solid_line_num=flows2[0].solid_line_num.np.astype(np.int32),
                        **before3, **after3, **before2, **after2)
    print(f"{name}: ok")


def _tool_kernels(R, path, names, extra_globals):
    """The @wp.kernel / @wp.func definitions ``names`` (and the module-level ``_LIVE*`` constants)
    of a reference tool script, executed under the emulator without importing the script (its
    imports pull in OpenGL, OpenCV and MuJoCo, which the kernels do not use)."""
    import ast

    src = open(path).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body
            if (isinstance(n, ast.FunctionDef) and n.name in names)
            or (isinstance(n, ast.Assign) and all(isinstance(t, ast.Name) and t.id.startswith("_LIVE")
                                                  for t in n.targets))]
    mod = ast.Module(body=keep, type_ignores=[])
    ns = dict(extra_globals)
    ns.update({"wp": R.wp, "np": np, "math": __import__("math")})
    # dont_inherit: this script's own `from __future__ import annotations` would turn the kernels'
    # annotations into strings, and the emulator converts scalar arguments by annotation type
    exec(compile(mod, path, "exec", dont_inherit=True), ns)
    return ns


def case_diagnostics(R, name, seed):
    """The display kernels on random fields: 2D get_u_img, get_velocity_rgb, get_vorticity_img,
    get_vorticity_with_solid_img, get_solid_boundary_img (envs/lbm/lbm_func.py:163-319, 804-866);
    3D slices and projections with mesh silhouettes (envs/lbm3d/lbm_func_3d.py:753-842, 990-1313);
    the live 3D view's slice stack and colour map (tools/lbm3d_realtime_control.py:68-182); the
    2D tool's image colour map and force brush (tools/lbm2d_realtime_control.py:144-157, 417-464).
    The 3D *_with_solid slices are left out: their inside test is Warp's native
    mesh_query_point_sign_normal, which the emulator does not restate."""
    wp = R.wp
    rng = np.random.default_rng(seed)
    out = {}
    # ---- 2D
    nx, ny = 26, 19
    f2 = R.core2.HomeFlow()
    f2.Initialize(nx, ny, n_objects=2)
    square = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float32)
    circle = np.asarray(R.solid.generate_unit_circle_points(12), np.float32)
    f2.configure_solid(0, square, (7.3, 8.6), angle=0.35, scale=2.2 / nx)
    f2.configure_solid(1, circle, (17.8, 10.1), angle=0.0, scale=2.9 / nx)
    fw2 = wp.array([f2], dtype=R.core2.HomeFlow)
    wp.launch(R.func2.InitBoundary, dim=(1, nx, ny), inputs=[fw2])
    m = np.zeros((6, nx, ny), np.float32)
    m[0] = 1.0
    m[1] = rng.uniform(-0.06, 0.06, (nx, ny))
    m[2] = rng.uniform(-0.06, 0.06, (nx, ny))
    _set_moments2d(f2, m)
    wp.launch(R.func2.precompute_transformed_segments, dim=(1, 2, f2.max_segments_per_object), inputs=[fw2])
    out["u2"] = m[1:3].copy()
    out["line_tf2"] = f2.solid_line_transformed.np.copy()
    out["line_num2"] = f2.solid_line_num.np.astype(np.int32)
    out["position2"] = f2.solid_position.np.copy()
    out["scale2"] = f2.solid_scale.np.copy()
    out["max_radius2"] = f2.solid_max_radius.np.copy()
    out["grid_length2"] = np.float32(f2.grid_length)
    wp.launch(R.func2.get_u_img, dim=(nx, ny), inputs=[f2])
    out["u_img"] = f2.u_img.np.copy()
    wp.launch(R.func2.get_velocity_rgb, dim=(nx, ny), inputs=[f2, 0.05])
    out["velocity_rgb"] = f2.u_img_rgb.np.copy()
    wp.launch(R.func2.get_vorticity_img, dim=(nx, ny), inputs=[f2])
    out["vorticity2"] = f2.u_img.np.copy()
    wp.launch(R.func2.get_vorticity_with_solid_img, dim=(nx, ny), inputs=[f2, 1.3])
    out["vorticity2_solid"] = f2.u_img.np.copy()
    wp.launch(R.func2.get_solid_boundary_img, dim=(nx, ny), inputs=[f2, 1.3])
    out["solid_boundary2"] = f2.u_img.np.copy()
    # ---- 2D tool kernels
    t2 = _tool_kernels(R, os.path.join(R.root, "tools", "lbm2d_realtime_control.py"),
                       {"lbm_uimg_to_rgba_kernel", "set_local_force_kernel", "_clamp01"},
                       {"HomeFlow": R.core2.HomeFlow})
    for mode, img_key, vmax in ((0, "u_img", 0.06), (1, "vorticity2", 0.02), (2, "solid_boundary2", 1.0)):
        f2.u_img.np[...] = out[img_key]
        rgba = wp.zeros((ny, nx, 4), dtype=wp.uint8)
        wp.launch(t2["lbm_uimg_to_rgba_kernel"], dim=(nx, ny), inputs=[f2, rgba, mode, vmax])
        out[f"uimg_rgba_{mode}"] = rgba.np.copy()
    out["local_force_args"] = np.array([9.5, 7.25, 5.0, 3.5, 2e-4, -1e-4], np.float32)
    wp.launch(t2["set_local_force_kernel"], dim=(1, nx, ny), inputs=[fw2, *[float(v) for v in out["local_force_args"]]])
    out["local_force"] = np.stack([f2.forcex.np, f2.forcey.np]).copy()
    # ---- 3D
    shape = (14, 12, 10)
    f3 = R.core3.HomeFlow3D()
    f3.Initialize(*shape, n_objects=1)
    fw3 = wp.array([f3], dtype=R.core3.HomeFlow3D)
    wp.launch(R.func3.InitBoundary3D, dim=(1,) + shape, inputs=[fw3])
    m3 = _random_moments3d(rng, shape)
    m3[1:4] *= np.float32(1.5)
    _set_moments3d(f3, m3)
    verts, faces = _octahedron(3.1)
    mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3), indices=wp.array(faces.ravel(), dtype=wp.int32))
    f3.mesh_ids.np[0] = mesh.id
    f3.mesh_scale_sizes.np[0] = (1.0, 1.2, 0.9)
    q = _quat_wxyz((0.2, 1.0, 0.4), 0.7)
    f3.mesh_transforms.np[0] = (6.3, 5.6, 4.7, q[1], q[2], q[3], q[0])
    out["u3"] = m3[1:4].copy()
    out["flag3"] = f3.flag.np.copy()
    out["grid_length3"] = np.float32(f3.grid_length)
    out["mesh_vertices"], out["mesh_faces"] = verts, faces
    out["mesh_transform"] = f3.mesh_transforms.np[0].astype(np.float32).copy()
    out["mesh_scale"] = f3.mesh_scale_sizes.np[0].astype(np.float32).copy()
    nx3, ny3, nz3 = shape
    for kern, dim, arg, field, key in (
            (R.func3.get_u_img_xy_3d, (nx3, ny3), 6, "u_img_xy", "u_xy_6"),
            (R.func3.get_u_img_yz_3d, (ny3, nz3), 5, "u_img_xz", "u_yz_5"),
            (R.func3.get_vorticity_xy_3d, (nx3, ny3), 3, "u_img_xy", "vort_xy_3"),
            (R.func3.get_vorticity_yz_3d, (ny3, nz3), 9, "u_img_xz", "vort_yz_9")):
        wp.launch(kern, dim=dim, inputs=[f3, arg])
        out[key] = getattr(f3, field).np.copy()
    for kname, dim, field in (("get_u_projection_topdown_3d", (nx3, ny3), "u_img_xy"),
                              ("get_u_projection_max_topdown_3d", (nx3, ny3), "u_img_xy"),
                              ("get_vorticity_projection_topdown_3d", (nx3, ny3), "u_img_xy"),
                              ("get_u_projection_side_3d", (ny3, nz3), "u_img_xz"),
                              ("get_u_projection_front_3d", (nx3, nz3), "u_img_xz_front"),
                              ("get_vorticity_projection_side_3d", (ny3, nz3), "u_img_xz"),
                              ("get_vorticity_projection_front_3d", (nx3, nz3), "u_img_xz_front")):
        wp.launch(getattr(R.func3, kname), dim=dim, inputs=[f3])
        out[kname] = getattr(f3, field).np.copy()
    # ---- live slice stack
    t3 = _tool_kernels(R, os.path.join(R.root, "tools", "lbm3d_realtime_control.py"),
                       {"_extract_live_vorticity_slices", "_live_clamp01", "_live_vorticity_to_rgba"},
                       {"HomeFlow3D": R.core3.HomeFlow3D})
    out["live_bins"] = np.int32(t3["_LIVE_HISTOGRAM_BINS"])
    live = []
    for slice_axis, color_axis, stride, margin, positions in ((2, 2, 1, 1, (0, 4, 9)), (0, 1, 2, 0, (3, 13)),
                                                              (1, 0, 3, 2, (6,))):
        w_ = {0: ny3, 1: nx3, 2: nx3}[slice_axis]
        h_ = {0: nz3, 1: nz3, 2: ny3}[slice_axis]
        pw, ph = (w_ + stride - 1) // stride, (h_ + stride - 1) // stride
        pos = wp.array(np.array(positions, np.int32), dtype=wp.int32)
        vals = wp.zeros(len(positions) * ph * pw, dtype=wp.float32)
        hist = wp.zeros(int(t3["_LIVE_HISTOGRAM_BINS"]), dtype=wp.int32)
        wp.launch(t3["_extract_live_vorticity_slices"], dim=(pw, ph, len(positions)),
                  inputs=[f3, pos, vals, hist, pw, ph, stride, slice_axis, color_axis, margin, 1])
        rgba = wp.zeros(vals.np.size * 4, dtype=wp.uint8)
        wp.launch(t3["_live_vorticity_to_rgba"], dim=vals.np.size, inputs=[vals, rgba, 0.05, 0.8])
        live.append(dict(args=np.array([slice_axis, color_axis, stride, margin, pw, ph], np.int32),
                         positions=np.array(positions, np.int32), values=vals.np.copy(), hist=hist.np.copy(),
                         rgba=rgba.np.copy()))
    for k, d in enumerate(live):
        for kk, v in d.items():
            out[f"live{k}_{kk}"] = v
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: ok")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("HOMELBM_REFERENCE"),
                    help="the reference's source tree (default: $HOMELBM_REFERENCE)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.reference:
        ap.error("--reference (or HOMELBM_REFERENCE) is required")
    R = import_reference(args.reference)
    circle = np.asarray(R.solid.generate_unit_circle_points(24), np.float32)
    square = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float32)
    cases = {
        "d2q9_walls": lambda: case_2d(
            R, "d2q9_walls", 20, 12, 4, 11, 0.02, [0, 1, 1, 1],
            [[0.05, 0.01], [0.0, 0.0], [0.0, 0.0], [0.0, 0.0]], [], None, "random", 1e-4),
        "d2q9_bc_types": lambda: case_2d(
            R, "d2q9_bc_types", 14, 17, 4, 12, 0.05, [1, 0, 0, 2],
            [[0.0, 0.0], [0.03, -0.01], [-0.02, 0.02], [0.0, 0.0]], [], None, "random", 0.0),
        "d2q9_solids": lambda: case_2d(
            R, "d2q9_solids", 36, 22, 6, 13, 0.03, [0, 1, 1, 1],
            [[0.04, 0.0], [0.0, 0.0], [0.0, 0.0], [0.0, 0.0]],
            [dict(lines=circle, position=(11.3, 10.7), angle=0.0, scale=3.6 / 36),
             dict(lines=square, position=(24.6, 12.2), angle=0.3, scale=2.5 / 36)],
            [0.02, -0.01, 0.03], "uniform", 0.0),
        "d3q27_walls": lambda: case_3d(
            R, "d3q27_walls", (8, 7, 9), 3, 21, 0.05, [0, 1, 1, 0, 1, 2],
            [[0.03, 0.0, 0.01], [0, 0, 0], [0, 0, 0], [0.0, -0.02, 0.01], [0, 0, 0], [0, 0, 0]],
            force_amp=1e-4),
        "d3q27_periodic": lambda: case_3d(
            R, "d3q27_periodic", (6, 5, 7), 3, 22, 0.04, [1] * 6, [[0, 0, 0]] * 6, periodic=True,
            force_amp=1e-4),
        "d3q27_mesh": lambda: case_3d(
            R, "d3q27_mesh", (12, 11, 12), 3, 23, 0.05, [0, 1, 1, 1, 1, 1],
            [[0.03, 0.0, 0.0]] + [[0, 0, 0]] * 5,
            mesh=dict(radius=2.6, position=(5.7, 5.2, 6.1), velocity=(0.05, 0.02, -0.03),
                      axis=(0.3, 1.0, 0.2), omega=0.05)),
        "coupling": lambda: case_coupling(R, "coupling", 31),
        "init": lambda: case_init(R, "init"),
        "reset": lambda: case_reset(R, "reset", 41),
        "diagnostics": lambda: case_diagnostics(R, "diagnostics", 43),
    }
    for k, fn in cases.items():
        if args.only and k not in args.only.split(","):
            continue
        fn()
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "cases": sorted(cases)}, f, indent=1)


if __name__ == "__main__":
    main()
