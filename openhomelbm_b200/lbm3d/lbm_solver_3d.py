"""D3Q27 solver (drop-in for envs/lbm3d/lbm_solver_3d.py's LBM_Solver3D).

``step()`` advances every world by one step with the CUDA kernels of libhomelbm:
stream-collide (stream_and_collide_3d), the cut links and loads of the immersed meshes
(its narrow band and init_force_3d_batch), outer boundaries (apply_bc_3d) and the buffer
swap (Swap_Mom_3D). As in the reference (lbm_solver_3d.py:102-127) the first call
captures the step into a CUDA graph and later calls replay it; the graph is captured
once per buffer parity and again whenever viscosity, boundary conditions or buffers
change (the reference invalidates its graph the same way, karman_lbm_env_3d.py:280-305).
"""
from __future__ import annotations

import weakref
from typing import Any, Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _lib
from .._array import FlowArray, device_array, mask_tensor, reset as _reset
from .lbm_core_3d import HomeFlow3D


_BIN_CACHE: Dict[Tuple, Tuple] = {}


def triangle_bins(tris: np.ndarray, margin: float = 1.75, edge: float = 1.0, max_bins: int = 1 << 20):
    """Uniform grid of triangle lists over a body-frame mesh (T, 3, 3), for the link rays of
    the cut cells. Bin b lists every triangle whose bounding box, widened by ``margin`` (more
    than sqrt(3), the longest lattice link), meets b; the grid spans the mesh's bounding box
    widened the same way, so a ray of length <= sqrt(3) starting outside the grid hits nothing.
    Returns (origin x, y, z, edge), (nbx, nby, nbz), CSR starts (nbins + 1) and the lists.
    An empty mesh gives a 0 x 0 x 0 grid. Results are cached by mesh content."""
    if len(tris) == 0:
        return [0.0, 0.0, 0.0, 1.0], (0, 0, 0), np.zeros(1, np.int64), np.zeros(0, np.int64)
    t = np.ascontiguousarray(tris, np.float32)
    key = (t.shape, t.tobytes(), margin, edge, max_bins)
    hit = _BIN_CACHE.get(key)
    if hit is not None:
        return hit
    t = t.astype(np.float64)
    lo = t.min(axis=(0, 1)) - margin
    hi = t.max(axis=(0, 1)) + margin
    dims = np.maximum(np.ceil((hi - lo) / edge), 1).astype(np.int64)
    if dims.prod() > max_bins:
        edge *= (dims.prod() / max_bins) ** (1.0 / 3.0) * 1.001
        dims = np.maximum(np.ceil((hi - lo) / edge), 1).astype(np.int64)
    i0 = np.clip(np.floor((t.min(axis=1) - margin - lo) / edge).astype(np.int64), 0, dims - 1)
    i1 = np.clip(np.floor((t.max(axis=1) + margin - lo) / edge).astype(np.int64), 0, dims - 1)
    span = i1 - i0 + 1                       # (T, 3) bins per axis
    count = span.prod(axis=1)                # bins per triangle
    tri_ids = np.repeat(np.arange(len(t)), count)
    local = np.arange(count.sum()) - np.repeat(np.cumsum(count) - count, count)
    sy, sz = np.repeat(span[:, 1], count), np.repeat(span[:, 2], count)
    gx = np.repeat(i0[:, 0], count) + local // (sy * sz)
    gy = np.repeat(i0[:, 1], count) + (local // sz) % sy
    gz = np.repeat(i0[:, 2], count) + local % sz
    bins = (gx * dims[1] + gy) * dims[2] + gz
    order = np.lexsort((tri_ids, bins))
    bins, tri_ids = bins[order], tri_ids[order]
    start = np.searchsorted(bins, np.arange(dims.prod() + 1))
    out = ([float(lo[0]), float(lo[1]), float(lo[2]), float(edge)], tuple(int(d) for d in dims), start, tri_ids)
    if len(_BIN_CACHE) > 64:
        _BIN_CACHE.clear()
    _BIN_CACHE[key] = out
    return out


class LBM_Solver3D:
    """Advance one or more D3Q27 fluid worlds on a CUDA device."""

    def __init__(self, nx: int, ny: int, nz: int, solid_num: int = 1, nworld: int = 1,
                 device: Optional[Any] = None, *, storage: str = "float32", periodic: bool = False,
                 u_scale: float = 1.0, s_scale: float = 1.0, use_graph: bool = True, with_flag: bool = True,
                 with_force: bool = True) -> None:
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
        for k in range(self.nworld):
            f = HomeFlow3D()
            f.Initialize(nx, ny, nz, n_objects=solid_num, device=self.device, storage=storage,
                         u_scale=u_scale, s_scale=s_scale, periodic=periodic, with_flag=with_flag,
                         with_force=with_force)
            # the solver holds the meshes; the field diagnostics find them from the world (a
            # weak reference: a solver <-> world cycle would leave the solver, and the CUDA
            # graphs it holds, to the cyclic garbage collector, which may run during a capture)
            f.solver_ref, f.world_index = weakref.ref(self), k
            self.flows.append(f)
        stream = _lib.stream_ptr()
        L = _lib.lib()
        for f in self.flows:
            if not periodic and f.flag is not None:
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
        self._mesh_tris = [None] * self.solid_num
        self._tris = torch.zeros((1, 3, 3), dtype=torch.float32, device=self.device)
        self._tri_offset = torch.zeros(self.solid_num + 1, dtype=torch.int32, device=self.device)
        self._max_bound_radius = 0.0
        self._solid_version = 0
        self.use_bins = True
        self.use_work_list = True
        self._batch_solid_state()
        self.mujoco_mappings = {}
        self.mujoco_origins_wp = None
        self.lbm_origins_wp = None
        self.scales_wp = None
        self.solid_ids_wp = None
        self.solid_id_to_index = {}
        # the reference's flows_wp (lbm_solver_3d.py:68): the worlds as a device array
        self.flows_wp = FlowArray(self, 3)

    def _batch_solid_state(self) -> None:
        """Per-solid state of all worlds in batched tensors [nworld][n][...]; each world's
        HomeFlow3D fields are views of its row, so the coupling kernels address every world in
        one launch (the reference launches them over (nworld, n_solids) the same way)."""
        W, n, dev = self.nworld, self.solid_num, self.device
        f32 = dict(dtype=torch.float32, device=dev)
        self.solid_position_all = torch.zeros((W, n, 3), **f32)
        self.solid_quaternion_all = torch.zeros((W, n, 4), **f32)
        self.mesh_transforms_all = torch.zeros((W, n, 7), **f32)
        self.mesh_transforms_last_all = torch.zeros((W, n, 7), **f32)
        self.mesh_transforms_initialized_all = torch.zeros((W, n), dtype=torch.int32, device=dev)
        self.mesh_scale_sizes_all = torch.ones((W, n, 3), **f32)
        self.solid_bound_radius_all = torch.zeros((W, n), **f32)
        self.linear_v_all = torch.zeros((W, n, 3), **f32)
        self.angle_v_all = torch.zeros((W, n, 3), **f32)
        self.solid_force_all = torch.zeros((W, n, 3), **f32)
        self.solid_torque_all = torch.zeros((W, n, 3), **f32)
        self.loads64_all = torch.zeros((W, n, 6), dtype=torch.float64, device=dev)
        for w, f in enumerate(self.flows):
            # views of the batched rows; numpy() reads them back as wp.array.numpy() does
            f.solid_position = device_array(self.solid_position_all[w])
            f.solid_quaternion = device_array(self.solid_quaternion_all[w])
            f.mesh_transforms = device_array(self.mesh_transforms_all[w])
            f.mesh_transforms_last = device_array(self.mesh_transforms_last_all[w])
            f.mesh_transforms_initialized = device_array(self.mesh_transforms_initialized_all[w])
            f.mesh_scale_sizes = device_array(self.mesh_scale_sizes_all[w])
            f.solid_bound_radius = device_array(self.solid_bound_radius_all[w])
            f.linear_v = device_array(self.linear_v_all[w])
            f.angle_v = device_array(self.angle_v_all[w])
            f.solid_force = device_array(self.solid_force_all[w])
            f.solid_torque = device_array(self.solid_torque_all[w])
            f.loads64 = self.loads64_all[w]

    def _solids_struct(self, k: int) -> _lib.hl_solids3d:
        f = self.flows[k]
        s = _lib.hl_solids3d()
        s.n_objects = self.solid_num
        s.max_bound_radius = float(self._max_bound_radius)
        s.tri_offset = self._tri_offset.data_ptr()
        s.tris = self._tris.data_ptr()
        for name in ("transforms", "transforms_last"):
            setattr(s, name, getattr(f, "mesh_" + name).data_ptr())
        s.initialized = f.mesh_transforms_initialized.data_ptr()
        s.scale_sizes = f.mesh_scale_sizes.data_ptr()
        s.position = f.solid_position.data_ptr()
        s.bound_radius = f.solid_bound_radius.data_ptr()
        s.linear_v = f.linear_v.data_ptr()
        s.angle_v = f.angle_v.data_ptr()
        s.loads64 = f.loads64.data_ptr()
        s.force = f.solid_force.data_ptr()
        s.torque = f.solid_torque.data_ptr()
        if self.use_bins:
            s.bin_box = self._bin_box.data_ptr()
            s.bin_dims = self._bin_dims.data_ptr()
            s.bin_start = self._bin_start.data_ptr()
            s.bin_tris = self._bin_tris.data_ptr()
        if self.use_work_list:
            s.work = self._link_work[k].data_ptr()
        return s

    @property
    def has_meshes(self) -> bool:
        return any(t is not None and len(t) for t in self._mesh_tris)

    # ------------------------------------------------------------------ stepping
    def _launch(self, parity: int, stream, loads_out=None, stream_collide: bool = True,
                solid_links: bool = True) -> None:
        """One step of every world on ``stream``. ``loads_out`` (optional, per world a pair of
        device pointers) redirects the binary32 solid force / torque [n][3] of the step.
        ``stream_collide=False`` / ``solid_links=False`` leave out the stream-collide / cut-link
        launches (batched launches over several solvers' worlds, hl_d3q27_stream_collide_batch
        and hl_d3q27_solid_links_batch, do them); the boundaries always follow."""
        L = _lib.lib()
        meshes = self.has_meshes
        for k, f in enumerate(self.flows):
            w = f.world_struct(parity)
            diag = None
            if self.diagnostics:
                diag = _lib.hl_diag(self._diag_scratch[k].data_ptr(), self._diag_scratch[k].numel(),
                                    self.mass[k:k + 1].data_ptr(), self.health[k:k + 1].data_ptr())
            if stream_collide:
                _lib.check(L.hl_d3q27_stream_collide(w, float(f.vis_shear), diag, stream), "stream_and_collide_3d")
            if meshes and solid_links:
                sst = self._solids_struct(k)
                if loads_out is not None:
                    sst.force, sst.torque = loads_out[k]
                _lib.check(L.hl_d3q27_solid_links(w, float(f.vis_shear), sst, stream),
                           "stream_and_collide_3d (cut links)")
            if not f.periodic:
                _lib.check(L.hl_d3q27_apply_bc(w, f.bc_struct(), _lib.ptr(self._bc_scratch[k]), stream),
                           "apply_bc_3d")

    def _key(self):
        return tuple((float(f.vis_shear), tuple(map(int, f.bc_type)), f.bc_value.tobytes(), f.use_force,
                      tuple(m.data_ptr() for m in f.moments)) for f in self.flows) + (self.diagnostics,
                                                                                       self._solid_version)

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
        """One world's fluid field and transform history (lbm_solver_3d.py:348-365)."""
        self.reset_worlds([world_idx])

    def reset_worlds(self, world_indices: Sequence[int]) -> None:
        """Selected worlds' fluid fields and transform histories (lbm_solver_3d.py:367-385):
        ResetSingleWorldFlow3D over the mask of those worlds (rho = 1, u = 0, S = 0 in both buffers,
        body force zeroed) and mesh_transforms_initialized = 0, so the next pose update starts
        with zero wall velocity. One launch for all of them."""
        mask = np.zeros(self.nworld, np.int32)
        for i in world_indices:
            i = int(i)
            if not 0 <= i < self.nworld:
                raise ValueError(f"world index {i} out of range [0, {self.nworld})")
            mask[i] = 1
        self.reset_worlds_mask(mask, _lib.HL_RESET_FLOW | _lib.HL_RESET_INITIALIZED)

    def reset_worlds_mask(self, reset_mask, what: int = _lib.HL_RESET_FLOW | _lib.HL_RESET_INITIALIZED) -> None:
        """The masked resets over flows_wp (one entry per world, non-zero: reset) in one launch;
        ``what`` is a set of HL_RESET_* parts (default: what reset_worlds does)."""
        _reset(self.flows_wp, mask_tensor(reset_mask, self.nworld, self.device), what)

    # ------------------------------------------------------------------ solids
    def create_solid_from_mesh(self, solid_id: int, mesh: Any, lbm_position: Optional[Tuple[float, float, float]] = None,
                               lbm_scale: float = 0.15, init_quaternion: Tuple[float, float, float, float] = (1, 0, 0, 0),
                               mujoco_origin: Optional[np.ndarray] = None) -> Dict[str, Any]:
        """The same triangle-mesh solid in every world (lbm_solver_3d.py:128-226).

        ``mesh`` is anything with ``vertices`` (V, 3) and ``faces`` (F, 3) in the body frame
        (a trimesh.Trimesh, or a (vertices, faces) pair). The vertices are scaled by
        ``lbm_scale * nx`` and not recentred; ``bound_radius`` is the largest scaled vertex
        norm. The solid starts at ``lbm_position`` (default: the domain centre) with
        ``init_quaternion`` (w, x, y, z) and zero wall velocity.
        """
        sid = int(solid_id)
        if not 0 <= sid < self.solid_num:
            raise ValueError(f"solid_id {solid_id} out of range [0, {self.solid_num})")
        if isinstance(mesh, (tuple, list)):
            verts, faces = np.asarray(mesh[0], np.float64), np.asarray(mesh[1], np.int64)
            mesh_local = (verts.copy(), faces.copy())
        else:
            verts, faces = np.asarray(mesh.vertices, np.float64), np.asarray(mesh.faces, np.int64)
            mesh_local = mesh.copy() if hasattr(mesh, "copy") else mesh
        if verts.ndim != 2 or verts.shape[1] != 3 or (faces.size and (faces.ndim != 2 or faces.shape[1] != 3)):
            raise ValueError("mesh needs vertices (V, 3) and faces (F, 3)")
        lbm_scale_actual = float(lbm_scale) * self.nx
        scaled_vertices = verts * lbm_scale_actual
        if lbm_position is None:
            lbm_position = (self.nx * 0.5, self.ny * 0.5, self.nz * 0.5)
        self.meshes[sid] = mesh_local
        vertices = np.array(scaled_vertices, dtype=np.float32)
        bound_radius = float(np.linalg.norm(vertices, axis=1).max()) if len(vertices) else 0.0
        self._mesh_tris[sid] = vertices[faces] if faces.size else np.zeros((0, 3, 3), np.float32)
        self._upload_meshes()
        for f in self.flows:
            f.mesh_ids[sid] = sid + 1
            f.mesh_scale_sizes[sid] = 1.0
            f.solid_position[sid] = torch.tensor(np.asarray(lbm_position, np.float32), device=self.device)
            f.solid_quaternion[sid] = torch.tensor(np.asarray(init_quaternion, np.float32), device=self.device)
            f.solid_bound_radius[sid] = bound_radius
            self._update_mesh_transform(f, sid)
        if mujoco_origin is None:
            mujoco_origin = np.zeros(3, dtype=np.float32)
        self.mujoco_mappings[sid] = {"mujoco_origin": np.array(mujoco_origin, dtype=np.float32),
                                     "lbm_origin": np.array(lbm_position, dtype=np.float32),
                                     "scale": lbm_scale_actual}
        return {"mesh": mesh_local, "vertices": scaled_vertices, "scale": lbm_scale_actual,
                "lbm_position": lbm_position, "quaternion": init_quaternion}

    def _upload_meshes(self) -> None:
        tris = [t if t is not None else np.zeros((0, 3, 3), np.float32) for t in self._mesh_tris]
        counts = [len(t) for t in tris]
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        allt = np.concatenate(tris) if sum(counts) else np.zeros((1, 3, 3), np.float32)
        self._tris = torch.tensor(np.ascontiguousarray(allt, np.float32), device=self.device)
        self._tri_offset = torch.tensor(offs, device=self.device)
        boxes, dims, starts, lists = [], [], [], []
        first_bin = first_tri = 0
        for t in tris:
            box, d, start, lst = triangle_bins(t)
            boxes.append(box)
            dims.append([d[0], d[1], d[2], first_bin])
            starts.append(start + first_tri)
            lists.append(lst)
            first_bin += len(start)
            first_tri += len(lst)
        dev = self.device
        self._bin_box = torch.tensor(np.array(boxes, np.float32), device=dev)
        self._bin_dims = torch.tensor(np.array(dims, np.int32), device=dev)
        self._bin_start = torch.tensor(np.concatenate(starts).astype(np.int32), device=dev)
        self._bin_tris = torch.tensor(np.concatenate(lists + [np.zeros(1, np.int32)]).astype(np.int32), device=dev)
        radii = [float(np.linalg.norm(t.reshape(-1, 3), axis=1).max()) for t in tris if len(t)]
        self._max_bound_radius = max(radii) if radii else 0.0
        ints = int(_lib.lib().hl_d3q27_solid_links_work_ints(self.solid_num, float(self._max_bound_radius)))
        self._link_work = [torch.zeros(max(ints, 1), dtype=torch.int32, device=dev) for _ in self.flows]
        self._solid_version += 1

    def _update_mesh_transform(self, flow: HomeFlow3D, solid_id: int) -> None:
        """New mesh transform from solid_position / solid_quaternion (lbm_solver_3d.py:244-268):
        the first time both transforms are set (zero wall velocity), afterwards the current one
        becomes the last. Device-side (hl_couple3d_update_solids with the identity mapping), so
        no host synchronisation."""
        self._pose_update(flow.world_index, [solid_id], flow.solid_position[solid_id:solid_id + 1],
                          flow.solid_quaternion[solid_id:solid_id + 1], identity=True)

    def _pose_update(self, world_idx: int, solid_ids, positions, quaternions, identity: bool) -> None:
        """One launch of the pose-in kernel for one world: positions (n, 3) and quaternions (n, 4,
        w x y z) of the solids ``solid_ids``, mapped through each solid's MuJoCo mapping unless
        ``identity``; updates solid_position / solid_quaternion and the mesh transforms."""
        n = len(solid_ids)
        dev = self.device
        ids = torch.as_tensor(np.asarray(solid_ids, np.int32)).to(dev)
        pos = torch.as_tensor(positions, dtype=torch.float32).reshape(1, n, 3).to(dev).contiguous()
        quat = torch.as_tensor(quaternions, dtype=torch.float32).reshape(1, n, 4).to(dev).contiguous()
        mo = np.zeros((n, 3), np.float32)
        lo = np.zeros((n, 3), np.float32)
        sc = np.ones(n, np.float32)
        if not identity:
            for i, sid in enumerate(solid_ids):
                m = self.mujoco_mappings.get(int(sid))
                if m is not None:
                    mo[i], lo[i], sc[i] = m["mujoco_origin"], m["lbm_origin"], np.float32(m["scale"])
        mo_t, lo_t, sc_t = (torch.as_tensor(a).to(dev) for a in (mo, lo, sc))
        W, S = self.nworld, self.solid_num
        w = int(world_idx)
        L = _lib.lib()
        off3, off4, off7 = w * S * 3, w * S * 4, w * S * 7
        _lib.check(L.hl_couple3d_update_solids(
            1, S, n, _lib.ptr(ids), _lib.ptr(pos), _lib.ptr(quat), _lib.ptr(mo_t), _lib.ptr(lo_t), _lib.ptr(sc_t),
            _lib.ptr(self.solid_position_all.view(-1)[off3:]), _lib.ptr(self.solid_quaternion_all.view(-1)[off4:]),
            _lib.ptr(self.mesh_transforms_all.view(-1)[off7:]), _lib.ptr(self.mesh_transforms_last_all.view(-1)[off7:]),
            _lib.ptr(self.mesh_transforms_initialized_all.view(-1)[w * S:]), _lib.stream_ptr()),
            "update_solids_batch")

    def update_solids_batch(self, world_idx: int, solid_ids: Sequence[int], positions: np.ndarray,
                            quaternions: np.ndarray) -> None:
        """Poses of several solids of one world from MuJoCo positions (N, 3) and quaternions
        (N, 4) in (w, x, y, z) order (lbm_solver_3d.py:270-306): lattice position
        (pos - mujoco_origin) * scale + lbm_origin where the solid has a mapping (the position as
        given otherwise), and the mesh transforms, in one launch without host synchronisation."""
        positions = np.asarray(positions, np.float32).reshape(-1, 3)
        quaternions = np.asarray(quaternions, np.float32).reshape(-1, 4)
        if len(positions) != len(solid_ids) or len(quaternions) != len(solid_ids):
            raise ValueError("positions and quaternions need one row per solid id")
        for sid in solid_ids:
            if not 0 <= int(sid) < self.solid_num:
                raise ValueError(f"solid_id {sid} out of range [0, {self.solid_num})")
        self._pose_update(world_idx, list(solid_ids), positions, quaternions, identity=False)

    def get_forces_and_torques(self, world_idx: int, solid_ids: Optional[Sequence[int]] = None
                               ) -> Tuple[np.ndarray, np.ndarray]:
        """Forces and torques (N, 3) of a world's solids, divided by the mapping scale and its
        square where a MuJoCo mapping exists (lbm_solver_3d.py:294-333)."""
        if solid_ids is None:
            solid_ids = list(range(self.solid_num))
        flow = self.flows[world_idx]
        sf = flow.solid_force.detach().cpu().numpy()
        st = flow.solid_torque.detach().cpu().numpy()
        forces = np.zeros((len(solid_ids), 3), np.float32)
        torques = np.zeros((len(solid_ids), 3), np.float32)
        for i, sid in enumerate(solid_ids):
            if sid in self.mujoco_mappings:
                scale = self.mujoco_mappings[sid]["scale"]
                forces[i] = sf[sid] / scale
                torques[i] = st[sid] / (scale * scale)
            else:
                forces[i] = sf[sid]
                torques[i] = st[sid]
        return forces, torques

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
