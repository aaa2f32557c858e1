"""MuJoCo-Warp coupling kernels (drop-in for envs/lbm/lbm_fluid_env_func.py and
envs/lbm3d/lbm_fluid_env_3d_func.py).

Each function replaces one Warp kernel of the coupled environments and keeps its name and
argument meaning; the environments' ``wp.launch(kernel, dim=(nworld, n_solids), inputs=[...])``
becomes a call of the function with torch CUDA tensors (or anything exposing
``__cuda_array_interface__`` through ``torch.as_tensor``). The solvers keep per-solid state of
all worlds in batched tensors (``solid_position_all`` ...), so one launch serves every world,
as the reference's 2-D launch does. Every function enqueues on the current stream and
synchronises nothing, so a caller can capture it into the step's CUDA graph.
"""
from __future__ import annotations

import torch

from . import _lib


def _dev(t, dtype, shape=None, name="buffer"):
    t = torch.as_tensor(t)
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t


def _ids(ids, bound, name):
    # Checked on the device (a thread with an id outside [0, bound) writes nothing): a host
    # check would read the ids back and synchronise the stream.
    return _dev(ids, torch.int32, name=name)


def extract_body_states(xipos, xquat, body_ids, positions_out, quaternions_out) -> None:
    """extract_body_states / extract_body_states_3d: positions_out (nworld, nsel, 3) and
    quaternions_out (nworld, nsel, 4, w x y z) from xipos (nworld, nbody, 3) and xquat
    (nworld, nbody, 4)."""
    xipos = _dev(xipos, torch.float32, name="xipos")
    nworld, nbody = xipos.shape[0], xipos.shape[1]
    xquat = _dev(xquat, torch.float32, (nworld, nbody, 4), "xquat")
    ids = _ids(body_ids, nbody, "body_ids")
    nsel = ids.numel()
    po = _dev(positions_out, torch.float32, (nworld, nsel, 3), "positions_out")
    qo = _dev(quaternions_out, torch.float32, (nworld, nsel, 4), "quaternions_out")
    _lib.check(_lib.lib().hl_couple_body_states(nworld, nbody, nsel, _lib.ptr(xipos), _lib.ptr(xquat), _lib.ptr(ids),
                                                _lib.ptr(po), _lib.ptr(qo), _lib.stream_ptr()), "extract_body_states")


def _solver(x):
    """The solver behind ``x``: a solver itself, or its ``flows_wp`` (the reference passes
    ``lbm_solver.flows_wp`` as these kernels' first input)."""
    from ._array import FlowArray

    return x.solver if isinstance(x, FlowArray) else x


def _mapping(solver, solid_ids, mujoco_origins, lbm_origins, scales, dim):
    ids = _ids(solid_ids if solid_ids is not None else solver.solid_ids_wp, solver.solid_num, "solid_ids")
    nsel = ids.numel()
    mo = solver.mujoco_origins_wp if mujoco_origins is None else torch.as_tensor(mujoco_origins, device=solver.device)
    lo = solver.lbm_origins_wp if lbm_origins is None else torch.as_tensor(lbm_origins, device=solver.device)
    sc = solver.scales_wp if scales is None else torch.as_tensor(scales, device=solver.device)
    if mo is None or lo is None or sc is None:
        raise ValueError("coordinate mappings are missing: call finalize_mappings or pass them")
    mo = _dev(mo.to(torch.float32).reshape(nsel, -1)[:, :dim].contiguous(), torch.float32, (nsel, dim), "mujoco_origins")
    lo = _dev(lo.to(torch.float32).reshape(nsel, -1)[:, :dim].contiguous(), torch.float32, (nsel, dim), "lbm_origins")
    sc = _dev(sc.to(torch.float32).reshape(nsel).contiguous(), torch.float32, (nsel,), "scales")
    return ids, nsel, mo, lo, sc


def convert_and_update_solid_batch_3d(solver, solid_ids, mujoco_positions, mujoco_quaternions, mujoco_origins=None,
                                      lbm_origins=None, scales=None) -> None:
    """convert_and_update_solid_batch_3d on an LBM_Solver3D: lattice positions, quaternions and
    mesh transforms of the selected solids in every world (the current transform moves to
    mesh_transforms_last, which is also set on the first call). Mappings default to the
    solver's finalize_mappings arrays. ``solver`` may be the solver's ``flows_wp``."""
    solver = _solver(solver)
    ids, nsel, mo, lo, sc = _mapping(solver, solid_ids, mujoco_origins, lbm_origins, scales, 3)
    W = solver.nworld
    mp = _dev(mujoco_positions, torch.float32, (W, nsel, 3), "mujoco_positions")
    mq = _dev(mujoco_quaternions, torch.float32, (W, nsel, 4), "mujoco_quaternions")
    _lib.check(_lib.lib().hl_couple3d_update_solids(
        W, solver.solid_num, nsel, _lib.ptr(ids), _lib.ptr(mp), _lib.ptr(mq), _lib.ptr(mo), _lib.ptr(lo), _lib.ptr(sc),
        _lib.ptr(solver.solid_position_all), _lib.ptr(solver.solid_quaternion_all),
        _lib.ptr(solver.mesh_transforms_all), _lib.ptr(solver.mesh_transforms_last_all),
        _lib.ptr(solver.mesh_transforms_initialized_all), _lib.stream_ptr()), "convert_and_update_solid_batch_3d")


def convert_and_update_solid_batch_2d(solver, solid_ids, mujoco_positions, mujoco_quaternions, mujoco_origins=None,
                                      lbm_origins=None, scales=None) -> None:
    """convert_and_update_solid_batch_2d on an LBM_Solver: planar positions and yaw angles of the
    selected solids in every world. ``solver`` may be the solver's ``flows_wp``."""
    solver = _solver(solver)
    ids, nsel, mo, lo, sc = _mapping(solver, solid_ids, mujoco_origins, lbm_origins, scales, 2)
    W = solver.nworld
    mp = _dev(mujoco_positions, torch.float32, (W, nsel, 3), "mujoco_positions")
    mq = _dev(mujoco_quaternions, torch.float32, (W, nsel, 4), "mujoco_quaternions")
    _lib.check(_lib.lib().hl_couple2d_update_solids(
        W, solver.solid_num, nsel, _lib.ptr(ids), _lib.ptr(mp), _lib.ptr(mq), _lib.ptr(mo), _lib.ptr(lo), _lib.ptr(sc),
        _lib.ptr(solver.solid_position_all), _lib.ptr(solver.solid_angle_all), _lib.stream_ptr()),
        "convert_and_update_solid_batch_2d")


def _loads(mode, solver, solid_ids, scales, fconv, tconv, forces_out, torques_out):
    solver = _solver(solver)
    ids = _ids(solid_ids, solver.solid_num, "solid_ids")
    nsel, W = ids.numel(), solver.nworld
    fo = _dev(forces_out, torch.float32, (W, nsel, 3), "forces_out")
    to = _dev(torques_out, torch.float32, (W, nsel, 3), "torques_out")
    sc = None if scales is None else _dev(torch.as_tensor(scales, device=solver.device).to(torch.float32).reshape(nsel)
                                          .contiguous(), torch.float32, (nsel,), "scales")
    if mode == 2:
        force, torque = solver.solid_loads_all, None
    else:
        force, torque = solver.solid_force_all, solver.solid_torque_all
    _lib.check(_lib.lib().hl_couple_loads(mode, W, solver.solid_num, nsel, _lib.ptr(ids), _lib.ptr(force),
                                          _lib.ptr(torque), _lib.ptr(sc), float(fconv), float(tconv), _lib.ptr(fo),
                                          _lib.ptr(to), _lib.stream_ptr()), "extract_forces_torques")


def extract_forces_torques_physical_3d(solver, solid_ids, force_conversion: float, torque_conversion: float,
                                       forces_out, torques_out) -> None:
    """Loads of the selected solids in physical units: force x rho dx^4 / dt^2, torque
    x rho dx^5 / dt^2 (the two conversion factors)."""
    _loads(0, solver, solid_ids, None, force_conversion, torque_conversion, forces_out, torques_out)


def extract_forces_torques_batch_3d(solver, solid_ids, scales, forces_out, torques_out) -> None:
    """Loads of the selected solids divided by the mapping scale (torque by its square)."""
    if scales is None:
        raise ValueError("scales are required")
    _loads(1, solver, solid_ids, scales, 1.0, 1.0, forces_out, torques_out)


def extract_forces_torques_batch(solver, solid_ids, scales, forces_out, torques_out) -> None:
    """Planar loads of an LBM_Solver as 3D MuJoCo loads: (fx, fy, 0) / scale and (0, 0, tz / scale)."""
    if scales is None:
        raise ValueError("scales are required")
    _loads(2, solver, solid_ids, scales, 1.0, 1.0, forces_out, torques_out)


def fill_xfrc(xfrc, body_ids, forces, torques) -> None:
    """fill_xfrc_kernel / fill_xfrc_3d_kernel: xfrc[w, body_ids[i]] = (forces[w, i], torques[w, i])
    in MuJoCo's spatial-force layout (force then torque); xfrc is (nworld, nbody, 6)."""
    xfrc = _dev(xfrc, torch.float32, name="xfrc")
    nworld, nbody = xfrc.shape[0], xfrc.shape[1]
    if xfrc.dim() != 3 or xfrc.shape[2] != 6:
        raise ValueError("xfrc must be (nworld, nbody, 6)")
    ids = _ids(body_ids, nbody, "body_ids")
    nsel = ids.numel()
    f = _dev(forces, torch.float32, (nworld, nsel, 3), "forces")
    t = _dev(torques, torch.float32, (nworld, nsel, 3), "torques")
    _lib.check(_lib.lib().hl_couple_fill_xfrc(nworld, nbody, nsel, _lib.ptr(ids), _lib.ptr(f), _lib.ptr(t),
                                              _lib.ptr(xfrc), _lib.stream_ptr()), "fill_xfrc")


fill_xfrc_kernel = fill_xfrc
fill_xfrc_3d_kernel = fill_xfrc
extract_body_states_3d = extract_body_states
