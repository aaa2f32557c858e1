"""The 2D realtime tool's interactive controls (tools/lbm2d_realtime_control.py:129-157) on a
solver's worlds: a boundary velocity, a prescribed solid motion, a local force region.

The reference runs each as a one-thread-per-world (or per-cell) Warp kernel over the worlds;
here the per-cell force field is a CUDA kernel (hl_d2q9_local_force) and the per-world values
are set directly: the boundary values are host state of each world (they go into the step's
launch arguments, so a change rebuilds the step's CUDA graph, as a change of viscosity does),
the solid poses are device tensors updated in place.
"""
from __future__ import annotations

from typing import Sequence

import torch

from .. import _lib


def set_boundary_velocity(flows: Sequence, boundary_idx: int, ux: float, uy: float) -> None:
    """set_boundary_velocity_kernel (129-133): bc_value[boundary_idx] = (ux, uy) in every world."""
    if not 0 <= int(boundary_idx) < 4:
        raise ValueError(f"boundary index {boundary_idx} outside 0..3")
    for f in flows:
        f.bc_value[int(boundary_idx)] = (float(ux), float(uy))


def advance_prescribed_solid_motion(flows: Sequence, solid_id: int, vx: float, vy: float, omega: float) -> None:
    """advance_prescribed_solid_motion_kernel (136-141): the solid's position moves by (vx, vy)
    and its angle by omega in every world."""
    for f in flows:
        if not 0 <= int(solid_id) < f.solid_position.shape[0]:
            raise ValueError(f"solid_id {solid_id} out of range [0, {f.solid_position.shape[0]})")
        f.solid_position[int(solid_id)] += torch.tensor((float(vx), float(vy)), dtype=f.solid_position.dtype,
                                                        device=f.solid_position.device)
        f.solid_angle[int(solid_id)] += float(omega)


def set_local_force(flows: Sequence, cx: float, cy: float, rx: float, ry: float, fx: float, fy: float) -> None:
    """set_local_force_kernel (144-157): every world's force field becomes
    (fx, fy) * max(0, 1 - ((x - cx)/rx)^2 - ((y - cy)/ry)^2), and its step uses it."""
    for f in flows:
        f.use_force = True
        _lib.check(_lib.lib().hl_d2q9_local_force(
            f.force[0].data_ptr(), f.force[1].data_ptr(), f.nx, f.ny, float(cx), float(cy), float(rx), float(ry),
            float(fx), float(fy), _lib.stream_ptr()), "local force")
