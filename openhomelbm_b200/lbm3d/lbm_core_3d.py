"""D3Q27 world state on torch CUDA tensors (drop-in for envs/lbm3d/lbm_core_3d.py).

``HomeFlow3D`` keeps the reference's field names and shapes (lbm_core_3d.py:44-136):
``rho`` (nx, ny, nz), ``u`` (nx, ny, nz, 3), ``Sxx`` ... ``Syz`` and their ``*_post`` twins,
``flag``, ``forcex/forcey/forcez`` and the per-solid arrays. Storage differs in one way
that callers do not see: the ten moments of a buffer are one SoA allocation
``(10, nx, ny, nz)`` (plane order rho, ux, uy, uz, Sxx, Syy, Szz, Sxy, Sxz, Syz) so that
the step kernel streams each plane with coalesced loads; ``u`` is a strided view. The two
buffers swap by a parity bit instead of by exchanging handles (Swap_Mom_3D, 689-727).
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .. import _lib
from .._array import device_array

# D3Q27 lattice in the reference's order (lbm_core_3d.py:12-35)
CX = (0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1)
CY = (0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1)
CZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1)
W = (8 / 27,) + (2 / 27,) * 6 + (1 / 54,) * 12 + (1 / 216,) * 8
INV = (0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25)
cs2 = 1.0 / 3.0
ML_FLUID, ML_SOLID, ML_WALL = 0, 1, 2

MOMENT_PLANES = ("rho", "ux", "uy", "uz", "Sxx", "Syy", "Szz", "Sxy", "Sxz", "Syz")
_S_PLANE = {"Sxx": 4, "Syy": 5, "Szz": 6, "Sxy": 7, "Sxz": 8, "Syz": 9}


class HomeFlow3D:
    """D3Q27 fluid and immersed-mesh state of one 3D world."""

    def Initialize(self, nx: int, ny: int, nz: int, n_objects: int = 1, *, device=None,
                   storage: str = "float32", u_scale: float = 1.0, s_scale: float = 1.0,
                   periodic: bool = False, with_flag: bool = True, with_force: bool = True) -> None:
        """Allocate the fields (reference: HomeFlow3D.Initialize, lbm_core_3d.py:138-227).

        ``storage`` selects the moment storage type ("float32", "float16", "bfloat16",
        "float64"); reduced types store rho-1, u/u_scale and (S-uu)/s_scale. ``periodic``
        makes every cell fluid with periodic neighbours (no walls, no apply_bc_3d).
        ``with_flag=False`` skips the flag field (the border cells are the walls, as
        InitBoundary3D would set them) and ``with_force=False`` the body-force field: a
        resident domain that needs neither then holds only its two moment buffers.
        """
        dev = _lib.require_cuda(device)
        self.device = dev
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.n_objects = int(n_objects)
        self.time_step = 1.0
        self.grid_length = 1.0 / nx
        self.velocity_scale = self.time_step / self.grid_length
        self.vis_shear = 0.1
        self.bc_type = [1, 1, 1, 1, 1, 1]
        self.bc_value = np.zeros((6, 3), np.float32)
        self.periodic = bool(periodic)
        self.storage_code = _lib.DTYPES[storage]
        self.storage = storage
        self.u_scale, self.s_scale = float(u_scale), float(s_scale)
        tdt = _lib.torch_dtype(self.storage_code)
        shape = (10, self.nx, self.ny, self.nz)
        self.moments = [torch.zeros(shape, dtype=tdt, device=dev), torch.zeros(shape, dtype=tdt, device=dev)]
        self.parity = 0
        self.flag = torch.zeros((self.nx, self.ny, self.nz), dtype=torch.int32, device=dev) if with_flag else None
        self.force = (torch.zeros((3, self.nx, self.ny, self.nz), dtype=torch.float32, device=dev) if with_force
                      else None)
        self.use_force = False
        n = self.n_objects
        f32 = dict(dtype=torch.float32, device=dev)
        self.mass = torch.zeros(n, **f32)
        self.MoI = torch.zeros(n, **f32)
        self.mesh_ids = torch.zeros(n, dtype=torch.int64, device=dev)
        self.mesh_transforms = torch.zeros((n, 7), **f32)
        self.mesh_transforms_last = torch.zeros((n, 7), **f32)
        self.mesh_transforms_initialized = torch.zeros(n, dtype=torch.int32, device=dev)
        self.mesh_scale_sizes = torch.ones((n, 3), **f32)
        self.linear_v = torch.zeros((n, 3), **f32)
        self.angle_v = torch.zeros((n, 3), **f32)
        self.solid_force = torch.zeros((n, 3), **f32)
        self.solid_position = torch.zeros((n, 3), **f32)
        self.solid_torque = torch.zeros((n, 3), **f32)
        self.solid_quaternion = torch.zeros((n, 4), **f32)
        self.solid_inertia = torch.zeros((n, 3, 3), **f32)
        self.solid_inertia_inv = torch.zeros((n, 3, 3), **f32)
        self.solid_bound_radius = torch.zeros(n, **f32)
        self.n_dirs = 27
        self.lat_e = torch.tensor(np.stack([CX, CY, CZ], 1), **f32)
        self.lat_w = torch.tensor(W, **f32)
        self.lat_inv = torch.tensor(INV, dtype=torch.int32, device=dev)
        # reference Initialize: rho = 1, everything else 0, in both buffers
        for m in self.moments:
            m[0].fill_(1.0 if not self.encoded else 0.0)
        # the per-world fields callers read back with numpy(), as from Warp arrays
        for name in ("flag", "mass", "MoI", "mesh_ids", "mesh_transforms", "mesh_transforms_last",
                     "mesh_transforms_initialized", "mesh_scale_sizes", "linear_v", "angle_v", "solid_force",
                     "solid_position", "solid_torque", "solid_quaternion", "solid_inertia", "solid_inertia_inv",
                     "solid_bound_radius"):
            setattr(self, name, device_array(getattr(self, name)))

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
        """Swap_Mom_3D: the post buffer becomes current."""
        self.parity ^= 1

    def decoded(self, post: bool = False) -> torch.Tensor:
        """The ten physical moments (10, nx, ny, nz) in float32 (float64 for that storage)."""
        m = self.post if post else self.cur
        if not self.encoded:
            return m
        r = m.float()
        out = torch.empty_like(r)
        out[0] = r[0] + 1.0
        out[1:4] = r[1:4] * self.u_scale
        u = out[1:4]
        pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
        for k, (a, b) in enumerate(pairs):
            out[4 + k] = r[4 + k] * self.s_scale + u[a] * u[b]
        return out

    def _plane(self, k: int, post: bool) -> torch.Tensor:
        if self.encoded:
            return device_array(self.decoded(post)[k])
        return device_array((self.post if post else self.cur)[k])

    rho = property(lambda s: s._plane(0, False))
    rho_post = property(lambda s: s._plane(0, True))
    u = property(lambda s: device_array((s.decoded(False) if s.encoded else s.cur)[1:4].permute(1, 2, 3, 0)))
    u_post = property(lambda s: device_array((s.decoded(True) if s.encoded else s.post)[1:4].permute(1, 2, 3, 0)))
    Sxx = property(lambda s: s._plane(4, False))
    Syy = property(lambda s: s._plane(5, False))
    Szz = property(lambda s: s._plane(6, False))
    Sxy = property(lambda s: s._plane(7, False))
    Sxz = property(lambda s: s._plane(8, False))
    Syz = property(lambda s: s._plane(9, False))
    Sxx_post = property(lambda s: s._plane(4, True))
    Syy_post = property(lambda s: s._plane(5, True))
    Szz_post = property(lambda s: s._plane(6, True))
    Sxy_post = property(lambda s: s._plane(7, True))
    Sxz_post = property(lambda s: s._plane(8, True))
    Syz_post = property(lambda s: s._plane(9, True))
    forcex = property(lambda s: None if s.force is None else device_array(s.force[0]))
    forcey = property(lambda s: None if s.force is None else device_array(s.force[1]))
    forcez = property(lambda s: None if s.force is None else device_array(s.force[2]))

    # ------------------------------------------------------------------ ABI structs
    def world_struct(self, parity: Optional[int] = None) -> _lib.hl_world3d:
        p = self.parity if parity is None else parity
        w = _lib.hl_world3d()
        w.nx, w.ny, w.nz = self.nx, self.ny, self.nz
        w.storage = _lib.hl_storage(self.storage_code, self.u_scale, self.s_scale)
        w.cur = self.moments[p].data_ptr()
        w.post = self.moments[p ^ 1].data_ptr()
        w.flag = None if (self.periodic or self.flag is None) else self.flag.data_ptr()
        w.force = self.force.data_ptr() if (self.use_force and self.force is not None) else None
        w.periodic = int(self.periodic)
        return w

    def bc_struct(self) -> _lib.hl_bc3d:
        bc = _lib.hl_bc3d()
        for f in range(6):
            bc.bc_type[f] = int(self.bc_type[f])
            for k in range(3):
                bc.bc_value[f][k] = float(self.bc_value[f][k])
        return bc
