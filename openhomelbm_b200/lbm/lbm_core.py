"""D2Q9 world state on torch CUDA tensors (drop-in for envs/lbm/lbm_core.py).

``HomeFlow`` keeps the reference's field names and shapes (lbm_core.py:17-88): ``rho``
(nx, ny), ``u`` (nx, ny, 2), ``Sxx``, ``Syy``, ``Sxy`` and their ``*_post`` twins, ``flag``,
``forcex``, ``forcey``, ``vis_shear``, ``bc_type``, ``bc_value`` and the polygon-solid arrays
(``solid_line``, ``solid_line_transformed(_last)``, ``solid_position``, ``solid_angle``,
``solid_scale``, ``solid_mass_center``, ``solid_max_radius``, ``solid_forcex/forcey``,
``torque``, ``mass``, ``MoI``). The six moments of a buffer are one SoA allocation
``(6, nx, ny)`` (rho, ux, uy, Sxx, Syy, Sxy); ``u`` is a strided view; the buffers swap by a
parity bit.
"""
from __future__ import annotations

import math
from typing import Any, Optional

import numpy as np
import torch

from .. import _lib
from .._array import device_array

CX = (0, 1, -1, 0, 0, 1, -1, -1, 1)
CY = (0, 0, 0, 1, -1, 1, 1, -1, -1)
W = (4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36)
INV = (0, 2, 1, 4, 3, 7, 8, 5, 6)
ML_FLUID, ML_SOLID, ML_WALL, ML_INVALID = 0, 1, 2, 6


class HomeFlow:
    """D2Q9 fluid and polygon-solid state of one 2D world."""

    def Initialize(self, nx: int, ny: int, n_objects: int = 1, *, device=None, storage: str = "float32",
                   u_scale: float = 1.0, s_scale: float = 1.0, periodic: bool = False) -> None:
        """Allocate the fields (reference: HomeFlow.Initialize, lbm_core.py:90-170)."""
        dev = _lib.require_cuda(device)
        self.device = dev
        self.time_step = 1.0
        self.nx, self.ny = int(nx), int(ny)
        self.grid_length = 1.0 / nx
        self.velocity_scale = self.time_step / self.grid_length
        self.periodic = bool(periodic)
        self.storage_code = _lib.DTYPES[storage]
        self.storage = storage
        self.u_scale, self.s_scale = float(u_scale), float(s_scale)
        tdt = _lib.torch_dtype(self.storage_code)
        self.moments = [torch.zeros((6, self.nx, self.ny), dtype=tdt, device=dev) for _ in range(2)]
        for m in self.moments:
            m[0].fill_(0.0 if self.encoded else 1.0)
        self.parity = 0
        self.flag = torch.zeros((self.nx, self.ny), dtype=torch.int32, device=dev)
        self.force = torch.zeros((2, self.nx, self.ny), dtype=torch.float32, device=dev)
        self.use_force = False
        self.vis_shear = 0.01
        self.bc_type = [1, 1, 1, 1]
        self.bc_value = np.zeros((4, 2), np.float32)
        self.w_d2q9, self.cx_d2q9, self.cy_d2q9, self.indexd2q9Inv_gpu = W, CX, CY, INV
        n = int(n_objects)
        self.n_objects = n
        f32 = dict(dtype=torch.float32, device=dev)
        self.solid_forcex = torch.zeros(n, **f32)
        self.solid_forcey = torch.zeros(n, **f32)
        self.torque = torch.zeros(n, **f32)
        self.mass = torch.zeros(n, **f32)
        self.MoI = torch.zeros(n, **f32)
        self.solid_position = torch.zeros((n, 2), **f32)
        self.solid_angle = torch.zeros(n, **f32)
        self.solid_scale = torch.zeros(n, **f32)
        self.solid_mass_center = torch.zeros((n, 2), **f32)
        self.solid_max_radius = torch.zeros(n, **f32)
        self.solid_line_num = torch.zeros(n, dtype=torch.int32, device=dev)
        self.max_segments_per_object = 10
        self.solid_line = torch.zeros((n, 10, 2), **f32)
        self.solid_line_transformed = torch.zeros((n, 10, 2), **f32)
        self.solid_line_transformed_last = torch.zeros((n, 10, 2), **f32)
        self.loads64 = torch.zeros((n, 3), dtype=torch.float64, device=dev)
        self.band_box = torch.zeros(4, dtype=torch.int32, device=dev)
        self.version = 0
        # the per-world fields callers read back with numpy(), as from Warp arrays
        for name in ("flag", "solid_forcex", "solid_forcey", "torque", "mass", "MoI", "solid_position", "solid_angle",
                     "solid_scale", "solid_mass_center", "solid_max_radius", "solid_line_num", "solid_line",
                     "solid_line_transformed", "solid_line_transformed_last"):
            setattr(self, name, device_array(getattr(self, name)))

    # ------------------------------------------------------------------ solids
    def configure_solid(self, solid_id: int, lines: Any, position: Any, angle: float = 0.0, scale: float = 0.3,
                        mass: float = 100000.0, mass_center: Optional[Any] = None) -> None:
        """Configure one polygon solid (reference: HomeFlow.configure_solid, lbm_core.py:172-280).

        Raises:
            ValueError: if ``solid_id`` is outside ``[0, n_objects)``.
        """
        if solid_id < 0 or solid_id >= self.n_objects:
            raise ValueError(f"solid_id {solid_id} out of range [0, {self.n_objects})")
        if isinstance(lines, torch.Tensor):
            lines_np = lines.detach().cpu().numpy()
        else:
            lines_np = np.asarray(lines, dtype=np.float32)
        lines_np = np.asarray(lines_np, np.float32).reshape(-1, 2)
        nseg = len(lines_np)
        if nseg > self.max_segments_per_object:
            old = self.max_segments_per_object
            self.max_segments_per_object = nseg
            for name in ("solid_line", "solid_line_transformed", "solid_line_transformed_last"):
                t = torch.zeros((self.n_objects, nseg, 2), dtype=torch.float32, device=self.device)
                if name == "solid_line":
                    t[:, :old] = getattr(self, name)
                setattr(self, name, device_array(t))
        mc = (0.0, 0.0) if mass_center is None else (float(mass_center[0]), float(mass_center[1]))
        # conservative squared radius in normalised units (lbm_core.py:248-256)
        max_dist = 0.0
        for p in lines_np:
            d = ((p[0] - mc[0]) ** 2 + (p[1] - mc[1]) ** 2) ** 0.5
            max_dist = max(max_dist, d)
        max_radius = (max_dist + math.sqrt(2.0)) ** 2
        moi = float(mass) * (float(scale) * float(self.nx)) ** 2.0 / 8.0
        self.solid_line[solid_id, :nseg] = torch.tensor(lines_np, device=self.device)
        self.solid_line_num[solid_id] = nseg
        self.solid_position[solid_id] = torch.tensor([float(position[0]), float(position[1])], device=self.device)
        self.solid_mass_center[solid_id] = torch.tensor(mc, device=self.device)
        self.solid_max_radius[solid_id] = float(np.float32(max_radius))
        self.solid_angle[solid_id] = float(angle)
        self.solid_scale[solid_id] = float(scale)
        self.mass[solid_id] = float(mass)
        self.MoI[solid_id] = moi
        self.version += 1

    # ------------------------------------------------------------------ views
    @property
    def encoded(self) -> bool:
        return self.storage_code in (_lib.HL_F16, _lib.HL_BF16)

    @property
    def cur(self) -> torch.Tensor:
        return self.moments[self.parity]

    @property
    def post(self) -> torch.Tensor:
        return self.moments[self.parity ^ 1]

    def swap(self) -> None:
        """Swap_Mom (lbm_func.py:475-500): the post buffer becomes current."""
        self.parity ^= 1

    def decoded(self, post: bool = False) -> torch.Tensor:
        m = self.post if post else self.cur
        if not self.encoded:
            return m
        r = m.float()
        out = torch.empty_like(r)
        out[0] = r[0] + 1.0
        out[1:3] = r[1:3] * self.u_scale
        out[3] = r[3] * self.s_scale + out[1] * out[1]
        out[4] = r[4] * self.s_scale + out[2] * out[2]
        out[5] = r[5] * self.s_scale + out[1] * out[2]
        return out

    def _plane(self, k: int, post: bool) -> torch.Tensor:
        return device_array((self.decoded(post) if self.encoded else (self.post if post else self.cur))[k])

    rho = property(lambda s: s._plane(0, False))
    rho_post = property(lambda s: s._plane(0, True))
    u = property(lambda s: device_array((s.decoded(False) if s.encoded else s.cur)[1:3].permute(1, 2, 0)))
    u_post = property(lambda s: device_array((s.decoded(True) if s.encoded else s.post)[1:3].permute(1, 2, 0)))
    Sxx = property(lambda s: s._plane(3, False))
    Syy = property(lambda s: s._plane(4, False))
    Sxy = property(lambda s: s._plane(5, False))
    Sxx_post = property(lambda s: s._plane(3, True))
    Syy_post = property(lambda s: s._plane(4, True))
    Sxy_post = property(lambda s: s._plane(5, True))
    forcex = property(lambda s: device_array(s.force[0]))
    forcey = property(lambda s: device_array(s.force[1]))

    # ------------------------------------------------------------------ ABI structs
    def world_struct(self) -> _lib.hl_world2d:
        w = _lib.hl_world2d()
        w.nx, w.ny = self.nx, self.ny
        w.storage = _lib.hl_storage(self.storage_code, self.u_scale, self.s_scale)
        w.cur = self.moments[0].data_ptr()
        w.post = self.moments[1].data_ptr()
        w.flag = None if self.periodic else self.flag.data_ptr()
        w.forcex = self.force[0].data_ptr() if self.use_force else None
        w.forcey = self.force[1].data_ptr() if self.use_force else None
        w.periodic = int(self.periodic)
        return w

    def step_struct(self) -> _lib.hl_step2d:
        return _lib.hl_step2d(float(self.vis_shear), float(self.grid_length), float(self.time_step))

    def bc_struct(self) -> _lib.hl_bc2d:
        bc = _lib.hl_bc2d()
        for f in range(4):
            bc.bc_type[f] = int(self.bc_type[f])
            bc.bc_value[f][0] = float(self.bc_value[f][0])
            bc.bc_value[f][1] = float(self.bc_value[f][1])
        return bc

    def solids_struct(self) -> Optional[_lib.hl_solids2d]:
        if self.n_objects == 0 or int(self.solid_line_num.max().item()) == 0:
            return None
        s = _lib.hl_solids2d()
        s.n_objects = self.n_objects
        s.max_segments = self.max_segments_per_object
        s.line = self.solid_line.data_ptr()
        s.line_num = self.solid_line_num.data_ptr()
        s.line_tf = self.solid_line_transformed.data_ptr()
        s.line_tf_last = self.solid_line_transformed_last.data_ptr()
        s.position = self.solid_position.data_ptr()
        s.angle = self.solid_angle.data_ptr()
        s.scale = self.solid_scale.data_ptr()
        s.mass_center = self.solid_mass_center.data_ptr()
        s.max_radius = self.solid_max_radius.data_ptr()
        s.loads64 = self.loads64.data_ptr()
        s.force_x = self.solid_forcex.data_ptr()
        s.force_y = self.solid_forcey.data_ptr()
        s.torque = self.torque.data_ptr()
        s.band_box = self.band_box.data_ptr()
        return s
