"""D3Q27 solver (drop-in for envs/lbm3d/lbm_solver_3d.py's LBM_Solver3D).

``step()`` advances every world by one step with the CUDA kernels of libhomelbm:
stream-collide (stream_and_collide_3d), outer boundaries (apply_bc_3d) and the buffer
swap (Swap_Mom_3D). As in the reference (lbm_solver_3d.py:102-127) the first call
captures the step into a CUDA graph and later calls replay it; the graph is captured
once per buffer parity and again whenever viscosity, boundary conditions or buffers
change (the reference invalidates its graph the same way, karman_lbm_env_3d.py:280-305).
"""
from __future__ import annotations

from typing import Any, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _lib
from .lbm_core_3d import HomeFlow3D


class LBM_Solver3D:
    """Advance one or more D3Q27 fluid worlds on a CUDA device."""

    def __init__(self, nx: int, ny: int, nz: int, solid_num: int = 1, nworld: int = 1,
                 device: Optional[Any] = None, *, storage: str = "float32", periodic: bool = False,
                 u_scale: float = 1.0, s_scale: float = 1.0, use_graph: bool = True) -> None:
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.solid_num = int(solid_num)
        self.nworld = int(nworld)
        self.device = _lib.require_cuda(device)
        self.captured = False
        self.captured_graph = None
        self.use_graph = use_graph
        self._graphs = {}
        self._graph_key = None
        self.flows = []
        for _ in range(self.nworld):
            f = HomeFlow3D()
            f.Initialize(nx, ny, nz, n_objects=solid_num, device=self.device, storage=storage,
                         u_scale=u_scale, s_scale=s_scale, periodic=periodic)
            self.flows.append(f)
        stream = _lib.stream_ptr()
        L = _lib.lib()
        for f in self.flows:
            if not periodic:
                _lib.check(L.hl_d3q27_init_boundary(f.nx, f.ny, f.nz, _lib.ptr(f.flag), stream),
                           "InitBoundary3D")
            _lib.check(L.hl_d3q27_init_uniform(f.nx, f.ny, f.nz, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                               _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), _lib.ptr(f.force),
                                               0.0, 0.0, 0.0, stream), "InitFlow3D")
        w0 = self.flows[0].world_struct()
        self._bc_scratch = [torch.zeros(int(L.hl_d3q27_bc_scratch_bytes(w0)), dtype=torch.uint8,
                                        device=self.device) for _ in self.flows]
        self._diag_scratch = [torch.zeros(int(L.hl_d3q27_scratch_bytes(w0)), dtype=torch.uint8,
                                          device=self.device) for _ in self.flows]
        self.mass = torch.zeros(self.nworld, dtype=torch.float64, device=self.device)
        self.health = torch.zeros(self.nworld, dtype=torch.int32, device=self.device)
        self.diagnostics = False
        self.meshes = [None] * self.solid_num
        self.mujoco_mappings = {}
        self.mujoco_origins_wp = None
        self.lbm_origins_wp = None
        self.scales_wp = None
        self.solid_ids_wp = None
        self.solid_id_to_index = {}

    # ------------------------------------------------------------------ stepping
    def _launch(self, parity: int, stream) -> None:
        L = _lib.lib()
        for k, f in enumerate(self.flows):
            w = f.world_struct(parity)
            diag = None
            if self.diagnostics:
                diag = _lib.hl_diag(self._diag_scratch[k].data_ptr(), self._diag_scratch[k].numel(),
                                    self.mass[k:k + 1].data_ptr(), self.health[k:k + 1].data_ptr())
            _lib.check(L.hl_d3q27_stream_collide(w, float(f.vis_shear), diag, stream), "stream_and_collide_3d")
            if not f.periodic:
                _lib.check(L.hl_d3q27_apply_bc(w, f.bc_struct(), _lib.ptr(self._bc_scratch[k]), stream),
                           "apply_bc_3d")

    def _key(self):
        return tuple((float(f.vis_shear), tuple(map(int, f.bc_type)), f.bc_value.tobytes(), f.use_force,
                      tuple(m.data_ptr() for m in f.moments)) for f in self.flows) + (self.diagnostics,)

    def step(self) -> None:
        """Advance every world by one LBM step (reference: LBM_Solver3D.step, 88-127)."""
        parity = self.flows[0].parity
        if not self.use_graph:
            self._launch(parity, _lib.stream_ptr())
        else:
            key = self._key()
            if key != self._graph_key:
                self._graphs = {}
                self._graph_key = key
            g = self._graphs.get(parity)
            if g is None:
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._launch(parity, _lib.stream_ptr())
                self._graphs[parity] = g
            g.replay()
            self.captured = True
            self.captured_graph = g
        for f in self.flows:
            f.swap()

    def invalidate_graph(self) -> None:
        self._graphs = {}
        self._graph_key = None
        self.captured = False
        self.captured_graph = None

    # ------------------------------------------------------------------ state
    def set_viscosity(self, viscosity: float) -> None:
        """Set vis_shear in every world (Karman3DEnv.set_viscosity, karman_lbm_env_3d.py:280-305)."""
        value = float(viscosity)
        if not np.isfinite(value) or value <= 0.0:
            raise ValueError("viscosity must be finite and positive")
        for f in self.flows:
            f.vis_shear = value

    def init_tgv(self, u0: float) -> None:
        """Taylor-Green initial state in every world (periodic box)."""
        L = _lib.lib()
        for f in self.flows:
            _lib.check(L.hl_d3q27_init_tgv(f.nx, f.ny, f.nz, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                           _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), float(u0),
                                           _lib.stream_ptr()), "init_tgv")

    def set_uniform_flow(self, ux: float, uy: float, uz: float) -> None:
        """set_uniform_flow_3d_kernel (envs/lbm3d/karman/karman_lbm_env_3d.py:15-64)."""
        L = _lib.lib()
        for f in self.flows:
            _lib.check(L.hl_d3q27_init_uniform(f.nx, f.ny, f.nz, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                               _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), _lib.ptr(f.force),
                                               float(ux), float(uy), float(uz), _lib.stream_ptr()),
                       "set_uniform_flow_3d")

    def reset_world(self, world_idx: int) -> None:
        """ResetSingleWorldFlow3D for one world (lbm_solver_3d.py:348-365)."""
        self.reset_worlds([world_idx])

    def reset_worlds(self, world_indices: Sequence[int]) -> None:
        L = _lib.lib()
        for i in world_indices:
            f = self.flows[int(i)]
            _lib.check(L.hl_d3q27_init_uniform(f.nx, f.ny, f.nz, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                               _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), _lib.ptr(f.force),
                                               0.0, 0.0, 0.0, _lib.stream_ptr()), "ResetSingleWorldFlow3D")
            f.mesh_transforms_initialized.zero_()

    def finalize_mappings(self, solid_ids: Sequence[int]) -> None:
        """Coordinate-mapping arrays for batch coupling (lbm_solver_3d.py:387-418)."""
        self.n = len(solid_ids)
        mo, lo, sc = [], [], []
        for idx, sid in enumerate(solid_ids):
            if sid not in self.mujoco_mappings:
                raise ValueError(f"Solid {sid} not initialized")
            m = self.mujoco_mappings[sid]
            mo.append(m["mujoco_origin"])
            lo.append(m["lbm_origin"])
            sc.append(m["scale"])
            self.solid_id_to_index[sid] = idx
        dev = self.device
        self.mujoco_origins_wp = torch.tensor(np.array(mo, np.float32), device=dev)
        self.lbm_origins_wp = torch.tensor(np.array(lo, np.float32), device=dev)
        self.scales_wp = torch.tensor(np.array(sc, np.float32), device=dev)
        self.solid_ids_wp = torch.tensor(list(solid_ids), dtype=torch.int32, device=dev)
