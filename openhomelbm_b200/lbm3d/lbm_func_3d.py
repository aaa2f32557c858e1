"""D3Q27 kernels that take ``flows_wp`` (drop-in for the reset kernels of envs/lbm3d/lbm_func_3d.py).

The reference launches them as ``wp.launch(Kernel, dim=(nworld, ...), inputs=[flows_wp,
reset_mask])``; here each is a function of the same name called as ``Kernel(flows_wp,
reset_mask)``. ``flows_wp`` is ``LBM_Solver3D.flows_wp``; ``reset_mask`` holds one entry per
world (non-zero: reset), as a CUDA int32 tensor (used in place, capturable) or anything numpy
accepts (copied to the device). Each call is one launch of hl_d3q27_reset_worlds on the current
stream; ``reset_worlds_masked`` does several parts in one launch.
"""
from __future__ import annotations

from .. import _lib
from .._array import reset as _reset


def ResetSingleWorldFlow3D(flows_wp, reset_mask) -> None:
    """lbm_func_3d.py:86-150: rho = 1, u = 0, S = 0 in both buffers and the body force zeroed in
    every masked world."""
    _reset(flows_wp, reset_mask, _lib.HL_RESET_FLOW)


def ResetSingleWorldSolidTransform3D(flows_wp, reset_mask) -> None:
    """lbm_func_3d.py:153-175: identity mesh transforms (current and last) and initialized = 0 for
    every solid of every masked world."""
    _reset(flows_wp, reset_mask, _lib.HL_RESET_SOLID_TRANSFORM)


def ResetSingleWorldForces3D(flows_wp, reset_mask) -> None:
    """lbm_func_3d.py:178-196: solid_force and solid_torque zeroed in every masked world."""
    _reset(flows_wp, reset_mask, _lib.HL_RESET_FORCES)


def reset_worlds_masked(flows_wp, reset_mask, flow: bool = True, solid_transform: bool = True,
                        forces: bool = True) -> None:
    """The three resets of partial_reset (envs/lbm3d/lbm_fluid_env_3d.py:578-611) in one launch."""
    what = ((_lib.HL_RESET_FLOW if flow else 0) | (_lib.HL_RESET_SOLID_TRANSFORM if solid_transform else 0) |
            (_lib.HL_RESET_FORCES if forces else 0))
    if what:
        _reset(flows_wp, reset_mask, what)
