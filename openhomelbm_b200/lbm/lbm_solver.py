"""D2Q9 solver (drop-in for envs/lbm/lbm_solver.py's LBM_Solver).

All worlds of a solver are stepped by one set of launches over a device array of world
descriptors (hl_d2q9_step_batch). The descriptors hold viscosity, boundary conditions and
buffer pointers and are re-uploaded whenever those change, so a captured CUDA graph stays
valid across parameter updates (the reference must rebuild ``flows_wp`` and recapture).
"""
from __future__ import annotations

from typing import Any, Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _lib
from .._array import FlowArray, device_array, mask_tensor, reset as _reset
from .lbm_core import HomeFlow


class LBM_Solver:
    """Advance one or more D2Q9 fluid worlds on a CUDA device (lbm_solver.py:21-244)."""

    def __init__(self, nx: int, ny: int, solid_num: int = 1, nworld: int = 1, device: Optional[Any] = None, *,
                 storage: str = "float32", periodic: bool = False, u_scale: float = 1.0, s_scale: float = 1.0,
                 use_graph: bool = True) -> None:
        self.nx, self.ny = int(nx), int(ny)
        self.solid_num = int(solid_num)
        self.nworld = int(nworld)
        self.device = _lib.require_cuda(device)
        self.captured = False
        self.captured_graph = None
        self.use_graph = use_graph
        self.flows = []
        for _ in range(self.nworld):
            f = HomeFlow()
            f.Initialize(nx, ny, n_objects=solid_num, device=self.device, storage=storage, u_scale=u_scale,
                         s_scale=s_scale, periodic=periodic)
            self.flows.append(f)
        # per-solid poses and loads of all worlds in batched tensors; each world's HomeFlow
        # fields are views of its row, so the coupling kernels serve every world in one launch
        W, n = self.nworld, self.solid_num
        f32 = dict(dtype=torch.float32, device=self.device)
        self.solid_position_all = torch.zeros((W, n, 2), **f32)
        self.solid_angle_all = torch.zeros((W, n), **f32)
        self.solid_loads_all = torch.zeros((W, 3, n), **f32)  # solid_forcex, solid_forcey, torque
        for w, f in enumerate(self.flows):
            # views of the batched rows; numpy() reads them back as wp.array.numpy() does
            f.solid_position = device_array(self.solid_position_all[w])
            f.solid_angle = device_array(self.solid_angle_all[w])
            f.solid_forcex = device_array(self.solid_loads_all[w, 0])
            f.solid_forcey = device_array(self.solid_loads_all[w, 1])
            f.torque = device_array(self.solid_loads_all[w, 2])
        self.total_steps = 500000
        self.per_frame_t = 500
        L = _lib.lib()
        st = _lib.stream_ptr()
        for f in self.flows:
            if not periodic:
                _lib.check(L.hl_d2q9_init_boundary(f.nx, f.ny, _lib.ptr(f.flag), st), "InitBoundary")
            _lib.check(L.hl_d2q9_init_uniform(f.nx, f.ny, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                              _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), _lib.ptr(f.force[0]),
                                              _lib.ptr(f.force[1]), 0.0, 0.0, st), "InitFlow")
        self._desc_bytes = int(L.hl_d2q9_desc_bytes())
        self._desc_dev = torch.zeros(self._desc_bytes * self.nworld, dtype=torch.uint8, device=self.device)
        self._desc_key = None
        self._graphs: Dict[Tuple, torch.cuda.CUDAGraph] = {}
        self.mujoco_mappings = {}
        self.mujoco_origins_wp = None
        self.lbm_origins_wp = None
        self.scales_wp = None
        self.solid_ids_wp = None
        self.solid_id_to_index = {}
        # the reference's flows_wp (lbm_solver.py:80): the worlds as a device array
        self.flows_wp = FlowArray(self, 2)

    def reset_worlds_mask(self, reset_mask, what: int = _lib.HL_RESET_FLOW | _lib.HL_RESET_SOLID_TRANSFORM |
                          _lib.HL_RESET_FORCES) -> None:
        """partial_reset's LBM part (envs/lbm/lbm_fluid_env.py:336-363) in one launch: for the
        worlds whose reset_mask entry is non-zero, ResetSingleWorldFlow, ResetSingleWorldSolidTransform
        and ResetSingleWorldForces (``what``: a set of HL_RESET_* parts)."""
        _reset(self.flows_wp, mask_tensor(reset_mask, self.nworld, self.device), what)

    # ------------------------------------------------------------------ descriptors
    def _params_key(self):
        return tuple((float(f.vis_shear), float(f.grid_length), float(f.time_step), tuple(map(int, f.bc_type)),
                      np.asarray(f.bc_value, np.float32).tobytes(), f.use_force, f.version,
                      f.solid_line.data_ptr(), int(f.parity)) for f in self.flows)

    def _upload_descriptors(self) -> None:
        L = _lib.lib()
        import ctypes

        host = bytearray(self._desc_bytes * self.nworld)
        base = (ctypes.c_char * len(host)).from_buffer(host)
        self._any_solid = False
        for k, f in enumerate(self.flows):
            s = f.solids_struct()
            self._any_solid |= s is not None
            _lib.check(L.hl_d2q9_pack(f.world_struct(), f.step_struct(), f.bc_struct(), s,
                                      ctypes.addressof(base) + k * self._desc_bytes), "pack world")
        self._desc_dev.copy_(torch.frombuffer(host, dtype=torch.uint8))

    def _launch(self, parity: int, stream) -> None:
        f0 = self.flows[0]
        _lib.check(_lib.lib().hl_d2q9_step_batch(_lib.ptr(self._desc_dev), self.nworld, parity, f0.storage_code,
                                                 self.nx, self.ny, int(self._any_solid), _lib.HL_PHASE_ALL,
                                                 stream), "LBM_Solver.step")

    def step(self) -> None:
        """Advance every world by one step (reference: LBM_Solver.step, lbm_solver.py:97-141)."""
        # every world's buffers start in the same parity (all are stepped together)
        parity = self.flows[0].parity
        key = self._params_key()
        desc_key = tuple(k[:-1] for k in key)
        if desc_key != self._desc_key:
            # a graph bakes only the descriptor array's address, so it stays valid
            self._upload_descriptors()
            self._desc_key = desc_key
        gkey = (parity, self._any_solid)
        if not self.use_graph:
            self._launch(parity, _lib.stream_ptr())
        else:
            g = self._graphs.get(gkey)
            if g is None:
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._launch(parity, _lib.stream_ptr())
                self._graphs[gkey] = g
            g.replay()
            self.captured = True
            self.captured_graph = g
        for f in self.flows:
            f.swap()

    # ------------------------------------------------------------------ solids / coupling
    def create_solid_from_polygon(self, solid_id: int, vertices: Any, lbm_position: Optional[Tuple[float, float]] = None,
                                  lbm_scale: float = 0.3, angle: float = 0.0,
                                  mujoco_origin: Optional[Sequence[float]] = None, **kwargs: Any) -> Dict[str, Any]:
        """Configure one polygon solid in every world and record its MuJoCo mapping.

        Same effect as ``create_solid_from_mujoco`` (lbm_solver.py:143-209) once the MuJoCo
        geometry has been projected to normalised polygon vertices.
        """
        if lbm_position is None:
            lbm_position = (self.nx * 0.5, self.ny * 0.5)
        for f in self.flows:
            f.configure_solid(solid_id=solid_id, lines=vertices, position=lbm_position, angle=angle,
                              scale=lbm_scale, **kwargs)
        self.mujoco_mappings[solid_id] = {
            "mujoco_origin": np.zeros(3, np.float32) if mujoco_origin is None else np.asarray(mujoco_origin, np.float32),
            "lbm_origin": np.array(lbm_position, dtype=np.float32),
            "scale": lbm_scale * self.nx,
        }
        return {"vertices": np.asarray(vertices, np.float32), "angle": angle}

    def create_solid_from_mujoco(self, solid_id: int, model: Any, data: Any, body_or_geom_name: str,
                                 lbm_position: Optional[Tuple[float, float]] = None, lbm_scale: Optional[float] = 0.3,
                                 n_samples: int = 20, is_body: bool = True, **kwargs: Any) -> Dict[str, Any]:
        """Project a MuJoCo body (or geom) into every world (lbm_solver.py:143-209).

        The outline comes from ``openhomelbm_b200.geometry.extract_lbm_polygon_from_mujoco``
        (convex hull, centred), or from a callable ``project(model, data, name, n_samples,
        is_body)`` returning {'vertices', 'angle', 'position'} passed as ``project=``. Returns
        the projection, as the reference does.
        """
        project = kwargs.pop("project", None)
        if project is None:
            from ..geometry import extract_lbm_polygon_from_mujoco

            info = extract_lbm_polygon_from_mujoco(model, data, body_or_geom_name, n_samples=n_samples,
                                                   use_convex_hull=True, normalize=True, is_body=is_body)
        else:
            info = project(model, data, body_or_geom_name, n_samples, is_body)
        self.create_solid_from_polygon(solid_id, info["vertices"], lbm_position, lbm_scale, info["angle"],
                                       mujoco_origin=info.get("position"), **kwargs)
        return info

    def finalize_mappings(self, solid_ids: Sequence[int]) -> None:
        """Coordinate-mapping arrays for batch coupling (lbm_solver.py:211-244)."""
        self.n = len(solid_ids)
        mo, lo, sc = [], [], []
        for idx, sid in enumerate(solid_ids):
            if sid not in self.mujoco_mappings:
                raise ValueError(f"Solid {sid} not initialized via create_solid_from_mujoco")
            m = self.mujoco_mappings[sid]
            mo.append(np.asarray(m["mujoco_origin"], np.float32)[:2])
            lo.append(np.asarray(m["lbm_origin"], np.float32)[:2])
            sc.append(m["scale"])
            self.solid_id_to_index[sid] = idx
        dev = self.device
        self.mujoco_origins_wp = torch.tensor(np.array(mo, np.float32), device=dev)
        self.lbm_origins_wp = torch.tensor(np.array(lo, np.float32), device=dev)
        self.scales_wp = torch.tensor(np.array(sc, np.float32), device=dev)
        self.solid_ids_wp = torch.tensor(list(solid_ids), dtype=torch.int32, device=dev)

    def set_uniform_flow(self, ux: float, uy: float) -> None:
        """set_uniform_flow_kernel (envs/lbm/karman/karman_lbm_env.py:15-53) in every world."""
        L = _lib.lib()
        for f in self.flows:
            _lib.check(L.hl_d2q9_init_uniform(f.nx, f.ny, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                              _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), _lib.ptr(f.force[0]),
                                              _lib.ptr(f.force[1]), float(ux), float(uy), _lib.stream_ptr()),
                       "set_uniform_flow")
