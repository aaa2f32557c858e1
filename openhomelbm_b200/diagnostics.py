"""Field diagnostics: headless images of a world's current fields (replaces the reference's
display kernels, envs/lbm/lbm_func.py:163-319, 804-866 and envs/lbm3d/lbm_func_3d.py:753-1313).

The functions keep the reference's kernel names and write the same fields of the world
(`u_img`, `u_img_rgb` for 2D; `u_img_xy` (nx, ny), `u_img_xz` (ny, nz), `u_img_xz_front`
(nx, nz) for 3D), allocated on first use as torch CUDA tensors; each also returns its image.
Everything runs on the world's device and current stream through `hl_d2q9_image` /
`hl_d3q27_image`; nothing reaches the host unless the caller copies it (a PNG, a video frame).
Where the reference launches `get_x(flow, ...)` with `wp.launch(..., dim=...)`, call `get_x(flow,
...)`.
"""
from __future__ import annotations

import torch

from . import _lib

U, RGB, VORTICITY, SOLIDS = 0, 1, 2, 3


def _buffer(flow, name: str, shape) -> torch.Tensor:
    t = getattr(flow, name, None)
    if not isinstance(t, torch.Tensor) or tuple(t.shape) != tuple(shape) or t.device != flow.device:
        t = torch.zeros(shape, dtype=torch.float32, device=flow.device)
        setattr(flow, name, t)
    return t


def _world2d(flow) -> _lib.hl_world2d:
    w = flow.world_struct()
    w.cur = flow.cur.data_ptr()  # the current buffer (world_struct describes the pair)
    return w


def _image2d(flow, kind: int, param: float = 0.0, thickness: float = 0.0, solids: bool = False) -> torch.Tensor:
    shape = (flow.nx, flow.ny, 3) if kind == RGB else (flow.nx, flow.ny)
    out = _buffer(flow, "u_img_rgb" if kind == RGB else "u_img", shape)
    s = flow.solids_struct() if solids else None
    _lib.check(_lib.lib().hl_d2q9_image(_world2d(flow), kind, float(param), float(flow.grid_length), s, float(thickness),
                                        out.data_ptr(), _lib.stream_ptr()), "field image")
    return out


# ------------------------------------------------------------------------------------ 2D
def get_u_img(flow) -> torch.Tensor:
    """|u| into flow.u_img (lbm_func.py:163-166)."""
    return _image2d(flow, U)


def get_velocity_rgb(flow, max_velocity: float) -> torch.Tensor:
    """(|u|, ux, uy) mapped from [-max, max] to [0, 1] into flow.u_img_rgb (169-193)."""
    if not max_velocity > 0:
        raise ValueError("max_velocity must be positive")
    return _image2d(flow, RGB, param=max_velocity)


def get_vorticity_img(flow) -> torch.Tensor:
    """dv/dx - du/dy into flow.u_img (196-233)."""
    return _image2d(flow, VORTICITY)


def get_vorticity_with_solid_img(flow, thickness: float) -> torch.Tensor:
    """Vorticity with the solids (inside or within `thickness`) marked 1000 (236-319)."""
    return _image2d(flow, VORTICITY, thickness=thickness, solids=True)


def get_solid_boundary_img(flow, thickness: float) -> torch.Tensor:
    """1 inside or within `thickness` of a solid, else 0, into flow.u_img (804-866)."""
    if flow.solids_struct() is None:
        out = _buffer(flow, "u_img", (flow.nx, flow.ny))
        out.zero_()
        return out
    return _image2d(flow, SOLIDS, thickness=thickness, solids=True)


# ------------------------------------------------------------------------------------ 3D
_PLANE = {2: ("u_img_xy", lambda f: (f.nx, f.ny)), 0: ("u_img_xz", lambda f: (f.ny, f.nz)),
          1: ("u_img_xz_front", lambda f: (f.nx, f.nz))}


def _image3d(flow, mode: int, axis: int, index: int, kind: int, thickness: float = 0.0,
             solids: bool = False) -> torch.Tensor:
    name, shape = _PLANE[axis]
    out = _buffer(flow, name, shape(flow))
    s = None
    ref = getattr(flow, "solver_ref", None)
    solver = ref() if ref is not None else None
    if solids and solver is not None and solver.has_meshes:
        s = solver._solids_struct(flow.world_index)
    _lib.check(_lib.lib().hl_d3q27_image(flow.world_struct(), mode, axis, int(index), kind, float(flow.grid_length), s,
                                         float(thickness), out.data_ptr(), _lib.stream_ptr()), "field image")
    return out


def get_u_img_xy_3d(flow, z_slice: int) -> torch.Tensor:
    """|u| on the plane z = z_slice into flow.u_img_xy (lbm_func_3d.py:753-761)."""
    return _image3d(flow, 0, 2, z_slice, 0)


def get_u_img_yz_3d(flow, x_slice: int) -> torch.Tensor:
    """|u| on the plane x = x_slice into flow.u_img_xz, shape (ny, nz) (764-776)."""
    return _image3d(flow, 0, 0, x_slice, 0)


def get_vorticity_xy_3d(flow, z_slice: int) -> torch.Tensor:
    """dv/dx - du/dy on z = z_slice into flow.u_img_xy (779-808)."""
    return _image3d(flow, 0, 2, z_slice, 1)


def get_vorticity_yz_3d(flow, x_slice: int) -> torch.Tensor:
    """dw/dy - dv/dz on x = x_slice into flow.u_img_xz (811-840)."""
    return _image3d(flow, 0, 0, x_slice, 1)


def get_vorticity_xy_with_solid_3d(flow, z_slice: int, thickness: float) -> torch.Tensor:
    """get_vorticity_xy_3d with solid voxels (flag, inside a mesh, within `thickness`) 1000 (843-911)."""
    return _image3d(flow, 0, 2, z_slice, 1, thickness, True)


def get_vorticity_yz_with_solid_3d(flow, x_slice: int, thickness: float) -> torch.Tensor:
    """get_vorticity_yz_3d with solid voxels 1000 (914-987)."""
    return _image3d(flow, 0, 0, x_slice, 1, thickness, True)


def get_u_projection_topdown_3d(flow) -> torch.Tensor:
    """|u| of the first moving cell seen from above (z high to low), mesh silhouettes 1000 (990-1030)."""
    return _image3d(flow, 1, 2, 0, 1, solids=True)


def get_u_projection_max_topdown_3d(flow) -> torch.Tensor:
    """max |u| along z, mesh silhouettes 1000 (1033-1069)."""
    return _image3d(flow, 1, 2, 0, 0, solids=True)


def get_vorticity_projection_topdown_3d(flow) -> torch.Tensor:
    """z vorticity of largest magnitude along z (sign kept), silhouettes 1000 (1072-1125)."""
    return _image3d(flow, 1, 2, 0, 2, solids=True)


def get_u_projection_side_3d(flow) -> torch.Tensor:
    """max |u| along x into flow.u_img_xz (ny, nz), silhouettes 1000 (1128-1163)."""
    return _image3d(flow, 1, 0, 0, 0, solids=True)


def get_u_projection_front_3d(flow) -> torch.Tensor:
    """max |u| along y into flow.u_img_xz_front (nx, nz), silhouettes 1000 (1166-1201)."""
    return _image3d(flow, 1, 1, 0, 0, solids=True)


def get_vorticity_projection_side_3d(flow) -> torch.Tensor:
    """x vorticity of largest magnitude along x into flow.u_img_xz (1204-1257)."""
    return _image3d(flow, 1, 0, 0, 2, solids=True)


def get_vorticity_projection_front_3d(flow) -> torch.Tensor:
    """y vorticity of largest magnitude along y into flow.u_img_xz_front (1260-1313)."""
    return _image3d(flow, 1, 1, 0, 2, solids=True)


# ----------------------------------------------------------------------------- live view
# The slice stack of the reference's live 3D view (tools/lbm3d_realtime_control.py:58-182,
# 820-869), on device buffers instead of a GL atlas.
_LIVE_HISTOGRAM_BINS = 256
_LIVE_LOG_VORT_MIN = -18.420680743952367  # log(1e-8)
_LIVE_LOG_VORT_MAX = 0.0                  # log(1.0)


def clear_live_histogram(histogram: torch.Tensor) -> None:
    """_clear_live_histogram: zero the 256 int32 bins."""
    histogram.zero_()


def extract_live_vorticity_slices(flow, slice_positions: torch.Tensor, values: torch.Tensor,
                                  histogram: torch.Tensor, plane_width: int, plane_height: int, stride: int,
                                  slice_axis: int, color_axis: int, boundary_margin: int,
                                  collect_histogram: int) -> None:
    """_extract_live_vorticity_slices (68-148): signed vorticity component `color_axis` on a
    stack of planes normal to `slice_axis` at `slice_positions` (int32, device), sampled every
    `stride` cells, into values[(slice * plane_height + q) * plane_width + p] (float32); with
    `collect_histogram`, the log-magnitude histogram of the nonzero values is added to
    `histogram` (int32, 256 bins)."""
    n = int(slice_positions.numel())
    for t, dt, need in ((slice_positions, torch.int32, n), (values, torch.float32, n * plane_width * plane_height),
                        (histogram, torch.int32, _LIVE_HISTOGRAM_BINS)):
        if t.dtype != dt or not t.is_cuda or not t.is_contiguous() or t.numel() < need:
            raise ValueError("live slices: slice_positions int32 (n), values float32 (n * width * height) and "
                             "histogram int32 (256), contiguous CUDA tensors")
    _lib.check(_lib.lib().hl_d3q27_live_slices(
        flow.world_struct(), slice_positions.data_ptr(), n, int(plane_width), int(plane_height), int(stride),
        int(slice_axis), int(color_axis), int(boundary_margin), int(collect_histogram), values.data_ptr(),
        histogram.data_ptr(), _lib.stream_ptr()), "live slices")


def live_vorticity_to_rgba(values: torch.Tensor, rgba: torch.Tensor, vmax: float, alpha: float) -> None:
    """_live_vorticity_to_rgba (157-182): blue-white-red map of values / vmax into rgba (uint8,
    4 per value)."""
    if values.dtype != torch.float32 or rgba.dtype != torch.uint8 or rgba.numel() < 4 * values.numel() \
            or not (values.is_cuda and rgba.is_cuda and values.is_contiguous() and rgba.is_contiguous()):
        raise ValueError("live rgba: values float32 and rgba uint8 (4 per value), contiguous CUDA tensors")
    _lib.check(_lib.lib().hl_live_rgba(values.data_ptr(), values.numel(), float(vmax), float(alpha), rgba.data_ptr(),
                                       _lib.stream_ptr()), "live rgba")


def vmax_from_histogram(counts, percentile: float, previous=None) -> float:
    """_update_vmax_from_histogram (820-831): the centre of the bin holding the `percentile`-th
    count, mapped back from log magnitude; 1e-6 for an empty histogram; against a previous
    value, the larger of it decayed by 0.96 and the new one (at least 1e-8). Host side."""
    import math

    import numpy as np

    counts = np.asarray(counts).astype(np.int64, copy=False)
    total = int(counts.sum())
    if total <= 0:
        current = 1.0e-6
    else:
        target = max(1, int(math.ceil(total * float(percentile) / 100.0)))
        bin_id = int(np.searchsorted(np.cumsum(counts), target, side="left"))
        fraction = (min(bin_id, _LIVE_HISTOGRAM_BINS - 1) + 0.5) / _LIVE_HISTOGRAM_BINS
        current = math.exp(_LIVE_LOG_VORT_MIN + fraction * (_LIVE_LOG_VORT_MAX - _LIVE_LOG_VORT_MIN))
    return max(current, 1.0e-8) if previous is None else max(previous * 0.96, current, 1.0e-8)


def lbm_uimg_to_rgba(flow, out: torch.Tensor, render_mode: int, vmax: float) -> torch.Tensor:
    """lbm_uimg_to_rgba_kernel (tools/lbm2d_realtime_control.py:417-464): flow.u_img (nx, ny)
    to RGBA bytes in `out` (uint8, (ny, nx, 4)); render_mode 0 velocity, 1 vorticity (solid
    marks grey), 2 solid boundary. A device buffer stands in for the GL pixel buffer."""
    img = getattr(flow, "u_img", None)
    if img is None or tuple(img.shape) != (flow.nx, flow.ny):
        raise ValueError("lbm_uimg_to_rgba: flow.u_img is not filled (call get_u_img or another 2D image first)")
    if out.dtype != torch.uint8 or tuple(out.shape) != (flow.ny, flow.nx, 4) or not out.is_contiguous() \
            or out.device != img.device:
        raise ValueError("lbm_uimg_to_rgba: out must be a contiguous uint8 (ny, nx, 4) tensor on the world's device")
    _lib.check(_lib.lib().hl_d2q9_uimg_rgba(img.data_ptr(), flow.nx, flow.ny, int(render_mode), float(vmax),
                                            out.data_ptr(), _lib.stream_ptr()), "uimg rgba")
    return out
