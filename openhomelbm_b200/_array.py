"""Device containers that keep the reference's host-side idioms working on torch CUDA tensors.

``DeviceArray`` is a CUDA tensor whose ``numpy()`` reads it back to the host, as
``wp.array.numpy()`` does for a Warp array on a GPU: the reference's callers read fields that
way (``flows[w].solid_position.numpy()[0]``, envs/lbm/eel/eel_lbm_env.py:126;
``flow.u_img.numpy().T``, envs/lbm/lbm_fluid_env.py:598), while a plain CUDA tensor's
``numpy()`` raises. Everything else is the tensor: the same storage, the same device pointer.

``FlowArray`` is the reference's ``flows_wp`` (``wp.array(self.flows, dtype=HomeFlow3D)``,
envs/lbm3d/lbm_solver_3d.py:68; ``HomeFlow``, envs/lbm/lbm_solver.py:80): it indexes like the
list of worlds, and holds the same worlds as one device array of world descriptors
(``hl_flow3d`` / ``hl_flow2d`` of include/homelbm.h) for the kernels that take ``flows_wp``
(the masked resets of ``lbm_func`` / ``lbm_func_3d``; the coupling functions take it in place
of the solver). The descriptor array is packed on first use and again whenever a world's
buffers move (creating or reshaping solids); that repacking copies from the host, so make the
first call of a kernel on ``flows_wp`` before capturing it into a CUDA graph.
"""
from __future__ import annotations

import ctypes
import weakref

import torch

from . import _lib


class DeviceArray(torch.Tensor):
    """A torch CUDA tensor whose ``numpy()`` copies it to host memory (``wp.array.numpy()``)."""

    def numpy(self, *args, **kwargs):  # noqa: D401 - same meaning as wp.array.numpy()
        return self.detach().as_subclass(torch.Tensor).cpu().numpy()


def device_array(t):
    """``t`` viewed as a DeviceArray (same storage), or None."""
    if t is None or isinstance(t, DeviceArray):
        return t
    return t.as_subclass(DeviceArray)


class FlowArray:
    """``flows_wp``: the worlds of a solver as a list and as a device array of descriptors."""

    def __init__(self, solver, dims: int) -> None:
        self._solver = weakref.ref(solver)  # no solver <-> array cycle (the solver holds CUDA graphs)
        self.dims = int(dims)
        self._key = None
        self._dev = None

    @property
    def solver(self):
        s = self._solver()
        if s is None:
            raise RuntimeError("flows_wp: its solver no longer exists")
        return s

    @property
    def flows(self):
        return self.solver.flows

    @property
    def device(self):
        return self.solver.device

    def __len__(self) -> int:
        return len(self.flows)

    def __getitem__(self, i):
        return self.flows[i]

    def __iter__(self):
        return iter(self.flows)

    @property
    def shape(self):
        return (len(self.flows),)

    def _structs(self):
        out = []
        for f in self.flows:
            sto = _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale)
            if self.dims == 3:
                d = _lib.hl_flow3d(f.nx, f.ny, f.nz, sto, f.moments[0].data_ptr(), f.moments[1].data_ptr(),
                                   None if f.force is None else f.force.data_ptr(), f.n_objects,
                                   f.mesh_transforms.data_ptr(), f.mesh_transforms_last.data_ptr(),
                                   f.mesh_transforms_initialized.data_ptr(), f.solid_force.data_ptr(),
                                   f.solid_torque.data_ptr())
            else:
                d = _lib.hl_flow2d(f.nx, f.ny, sto, f.moments[0].data_ptr(), f.moments[1].data_ptr(),
                                   f.force[0].data_ptr(), f.force[1].data_ptr(), f.n_objects,
                                   f.max_segments_per_object, f.solid_line_num.data_ptr(),
                                   f.solid_line_transformed.data_ptr(), f.solid_line_transformed_last.data_ptr(),
                                   f.solid_forcex.data_ptr(), f.solid_forcey.data_ptr(), f.torque.data_ptr())
            out.append(d)
        return out

    def descriptors(self) -> torch.Tensor:
        """The device array of world descriptors (uint8), repacked if any world's buffers moved."""
        structs = self._structs()
        raw = b"".join(bytes(memoryview(d)) for d in structs)
        if self._dev is None or raw != self._key:
            host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
            self._dev = host.to(self.device)
            self._key = raw
        return self._dev

    @property
    def ptr(self) -> int:
        return self.descriptors().data_ptr()

    def max_cells(self) -> int:
        """The launch extent the reset kernels need: the largest cell count of any world (2D:
        and its solids' outline points)."""
        m = 0
        for f in self.flows:
            cells = f.nx * f.ny * (f.nz if self.dims == 3 else 1)
            if self.dims == 2:
                cells = max(cells, f.n_objects * f.max_segments_per_object)
            m = max(m, cells)
        return m


def mask_tensor(reset_mask, nworld: int, device) -> torch.Tensor:
    """A reset mask as a contiguous int32 device tensor of nworld entries (non-zero: reset). A
    CUDA int32 tensor is used as it is (no copy, capturable); host masks are copied."""
    if isinstance(reset_mask, torch.Tensor) and reset_mask.is_cuda and reset_mask.dtype == torch.int32:
        m = reset_mask.reshape(-1)
        if not m.is_contiguous():
            m = m.contiguous()
    else:
        m = torch.as_tensor(reset_mask).reshape(-1).to(device=device, dtype=torch.int32)
    if m.numel() != nworld:
        raise ValueError(f"reset_mask has {m.numel()} entries for {nworld} worlds")
    return m


def reset(flows_wp: FlowArray, reset_mask, what: int) -> None:
    """One masked reset launch of the parts ``what`` (HL_RESET_* bits) over all worlds."""
    if not isinstance(flows_wp, FlowArray):
        raise TypeError("flows_wp must be a solver's flows_wp")
    n = len(flows_wp)
    m = mask_tensor(reset_mask, n, flows_wp.device)
    f0 = flows_wp[0]
    L = _lib.lib()
    fn = L.hl_d3q27_reset_worlds if flows_wp.dims == 3 else L.hl_d2q9_reset_worlds
    name = "ResetSingleWorld" + ("3D" if flows_wp.dims == 3 else "")
    _lib.check(fn(ctypes.c_void_p(flows_wp.ptr), n, f0.storage_code, ctypes.c_void_p(m.data_ptr()), int(what),
                  flows_wp.max_cells(), _lib.stream_ptr()), name)
