"""ctypes binding of libhomelbm.so (the C ABI declared in include/homelbm.h).

The library is the only compute path: if it cannot be loaded, or no CUDA device is
present, every entry point raises. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int, c_longlong, c_size_t,
                    c_void_p)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhomelbm.so")

HL_OK, HL_ERR_ARG, HL_ERR_UNSUPPORTED, HL_ERR_CUDA, HL_ERR_TIMEOUT = 0, -1, -2, -3, -4
HL_F32, HL_F16, HL_BF16, HL_F64 = 0, 1, 2, 3
HL_PHASE_SEGMENTS, HL_PHASE_STREAM, HL_PHASE_BC, HL_PHASE_ALL = 1, 2, 4, 7


class HomeLBMError(RuntimeError):
    """A CUDA-side failure reported by libhomelbm."""


class hl_storage(Structure):
    _fields_ = [("dtype", c_int), ("u_scale", c_float), ("s_scale", c_float)]


class hl_world3d(Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int), ("storage", hl_storage),
                ("cur", c_void_p), ("post", c_void_p), ("flag", c_void_p), ("force", c_void_p),
                ("periodic", c_int)]


class hl_bc3d(Structure):
    _fields_ = [("bc_type", c_int * 6), ("bc_value", (c_float * 3) * 6)]


class hl_diag(Structure):
    _fields_ = [("scratch", c_void_p), ("scratch_bytes", c_size_t), ("mass", c_void_p),
                ("health", c_void_p)]


class hl_solids3d(Structure):
    _fields_ = [("n_objects", c_int), ("max_bound_radius", c_float), ("tri_offset", c_void_p), ("tris", c_void_p),
                ("transforms", c_void_p), ("transforms_last", c_void_p), ("initialized", c_void_p),
                ("scale_sizes", c_void_p), ("position", c_void_p), ("bound_radius", c_void_p),
                ("linear_v", c_void_p), ("angle_v", c_void_p), ("loads64", c_void_p), ("force", c_void_p),
                ("torque", c_void_p), ("bin_box", c_void_p), ("bin_dims", c_void_p), ("bin_start", c_void_p),
                ("bin_tris", c_void_p), ("work", c_void_p)]


class hl_world2d(Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("storage", hl_storage), ("cur", c_void_p),
                ("post", c_void_p), ("flag", c_void_p), ("forcex", c_void_p), ("forcey", c_void_p),
                ("periodic", c_int)]


class hl_step2d(Structure):
    _fields_ = [("vis_shear", c_double), ("grid_length", c_float), ("time_step", c_float)]


class hl_bc2d(Structure):
    _fields_ = [("bc_type", c_int * 4), ("bc_value", (c_float * 2) * 4)]


class hl_solids2d(Structure):
    _fields_ = [("n_objects", c_int), ("max_segments", c_int), ("line", c_void_p),
                ("line_num", c_void_p), ("line_tf", c_void_p), ("line_tf_last", c_void_p),
                ("position", c_void_p), ("angle", c_void_p), ("scale", c_void_p),
                ("mass_center", c_void_p), ("max_radius", c_void_p), ("loads64", c_void_p),
                ("force_x", c_void_p), ("force_y", c_void_p), ("torque", c_void_p),
                ("band_box", c_void_p)]


class hl_flow3d(Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int), ("storage", hl_storage), ("m0", c_void_p),
                ("m1", c_void_p), ("force", c_void_p), ("n_objects", c_int), ("transforms", c_void_p),
                ("transforms_last", c_void_p), ("initialized", c_void_p), ("solid_force", c_void_p),
                ("solid_torque", c_void_p)]


class hl_flow2d(Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("storage", hl_storage), ("m0", c_void_p), ("m1", c_void_p),
                ("forcex", c_void_p), ("forcey", c_void_p), ("n_objects", c_int), ("max_segments", c_int),
                ("line_num", c_void_p), ("line_tf", c_void_p), ("line_tf_last", c_void_p),
                ("solid_forcex", c_void_p), ("solid_forcey", c_void_p), ("torque", c_void_p)]


HL_RESET_FLOW, HL_RESET_SOLID_TRANSFORM, HL_RESET_FORCES, HL_RESET_INITIALIZED = 1, 2, 4, 8

_lib = None

_SIGS = {
    "hl_last_error": ([], c_char_p),
    "hl_version": ([], c_char_p),
    "hl_set_tuning": ([c_char_p, c_int], c_int),
    "hl_d3q27_stream_collide": ([POINTER(hl_world3d), c_double, POINTER(hl_diag), c_void_p], c_int),
    "hl_d3q27_apply_bc": ([POINTER(hl_world3d), POINTER(hl_bc3d), c_void_p, c_void_p], c_int),
    "hl_d3q27_scratch_bytes": ([POINTER(hl_world3d)], c_size_t),
    "hl_d3q27_stream_collide_noalloc": ([POINTER(hl_world3d), c_double, c_void_p, c_void_p, c_void_p], c_int),
    "hl_d3q27_live_slices": ([POINTER(hl_world3d), c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                              c_void_p, c_void_p, c_void_p], c_int),
    "hl_live_rgba": ([c_void_p, c_longlong, c_float, c_float, c_void_p, c_void_p], c_int),
    "hl_round_to_storage": ([c_void_p, c_longlong, c_int, c_int, c_longlong, c_int, c_void_p, c_void_p], c_int),
    "hl_d2q9_uimg_rgba": ([c_void_p, c_int, c_int, c_int, c_float, c_void_p, c_void_p], c_int),
    "hl_d2q9_local_force": ([c_void_p, c_void_p, c_int, c_int, c_float, c_float, c_float, c_float, c_float, c_float,
                             c_void_p], c_int),
    "hl_d3q27_links_batch_bytes": ([c_int, c_int], c_size_t),
    "hl_d3q27_links_batch_prepare": ([POINTER(hl_world3d), POINTER(hl_solids3d), c_int, c_double, c_void_p, c_size_t,
                                      POINTER(c_size_t), c_void_p], c_int),
    "hl_d3q27_solid_links_batch": ([c_void_p, c_int, c_int, c_void_p, c_size_t, c_void_p], c_int),
    "hl_d3q27_batch_bytes": ([c_int], c_size_t),
    "hl_d3q27_batch_prepare": ([POINTER(hl_world3d), c_int, c_void_p, c_size_t, POINTER(c_int), c_void_p], c_int),
    "hl_d3q27_stream_collide_batch": ([c_void_p, c_int, c_int, c_double, POINTER(hl_storage), c_int, c_void_p,
                                       c_void_p], c_int),
    "hl_d3q27_bc_scratch_bytes": ([POINTER(hl_world3d)], c_size_t),
    "hl_d3q27_bc_batch_bytes": ([c_int], c_size_t),
    "hl_d3q27_bc_batch_prepare": ([POINTER(hl_world3d), POINTER(hl_bc3d), POINTER(c_void_p), c_int, c_void_p, c_size_t,
                                   c_void_p], c_int),
    "hl_d3q27_apply_bc_batch": ([c_void_p, c_int, c_int, c_void_p], c_int),
    "hl_d3q27_solid_links": ([POINTER(hl_world3d), c_double, POINTER(hl_solids3d), c_void_p], c_int),
    "hl_d3q27_solid_links_work_ints": ([c_int, c_float], c_size_t),
    "hl_couple_body_states": ([c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "hl_couple3d_update_solids": ([c_int, c_int, c_int] + [c_void_p] * 12, c_int),
    "hl_couple2d_update_solids": ([c_int, c_int, c_int] + [c_void_p] * 9, c_int),
    "hl_couple_loads": ([c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float,
                         c_void_p, c_void_p, c_void_p], c_int),
    "hl_couple_fill_xfrc": ([c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "hl_d3q27_init_uniform": ([c_int, c_int, c_int, hl_storage, c_void_p, c_void_p, c_void_p, c_float,
                               c_float, c_float, c_void_p], c_int),
    "hl_d3q27_init_tgv": ([c_int, c_int, c_int, hl_storage, c_void_p, c_void_p, c_float, c_void_p], c_int),
    "hl_d3q27_init_boundary": ([c_int, c_int, c_int, c_void_p, c_void_p], c_int),
    "hl_d2q9_step": ([POINTER(hl_world2d), POINTER(hl_step2d), POINTER(hl_bc2d), POINTER(hl_solids2d),
                      c_void_p], c_int),
    "hl_d2q9_step_phases": ([POINTER(hl_world2d), POINTER(hl_step2d), POINTER(hl_bc2d),
                             POINTER(hl_solids2d), c_int, c_void_p], c_int),
    "hl_d2q9_desc_bytes": ([], c_size_t),
    "hl_d2q9_pack": ([POINTER(hl_world2d), POINTER(hl_step2d), POINTER(hl_bc2d), POINTER(hl_solids2d),
                      c_void_p], c_int),
    "hl_d2q9_step_batch": ([c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p], c_int),
    "hl_d2q9_tile_shapes": ([c_void_p, c_int], c_int),
    "hl_d2q9_image": ([POINTER(hl_world2d), c_int, c_float, c_float, POINTER(hl_solids2d), c_float, c_void_p, c_void_p],
                      c_int),
    "hl_d3q27_image": ([POINTER(hl_world3d), c_int, c_int, c_int, c_int, c_float, POINTER(hl_solids3d), c_float, c_void_p,
                        c_void_p], c_int),
    "hl_d2q9_tile_list": ([c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_size_t, POINTER(c_size_t)], c_int),
    "hl_d2q9_step_tiles": ([c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int,
                            c_void_p], c_int),
    "hl_d2q9_init_uniform": ([c_int, c_int, hl_storage, c_void_p, c_void_p, c_void_p, c_void_p, c_float,
                              c_float, c_void_p], c_int),
    "hl_d2q9_init_boundary": ([c_int, c_int, c_void_p, c_void_p], c_int),
    "hl_d3q27_reset_worlds": ([c_void_p, c_int, c_int, c_void_p, c_int, c_longlong, c_void_p], c_int),
    "hl_d2q9_reset_worlds": ([c_void_p, c_int, c_int, c_void_p, c_int, c_longlong, c_void_p], c_int),
}


def declared_symbols():
    """Names of every function declared in include/homelbm.h (parsed from the header)."""
    import re

    with open(os.path.join(HERE, "..", "include", "homelbm.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hl_[a-z0-9_]+)\s*\(", text)))


def load(path: str = LIB_PATH):
    """Load libhomelbm.so and declare its signatures (no GPU needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise HomeLBMError(f"{path} is missing; build it with `python -m openhomelbm_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def lib():
    return load()


def check(rc: int, what: str = "") -> None:
    if rc != HL_OK:
        msg = lib().hl_last_error().decode(errors="replace")
        if rc == HL_ERR_ARG:
            raise ValueError(f"{what}: {msg}")
        if rc == HL_ERR_UNSUPPORTED:
            raise NotImplementedError(f"{what}: {msg}")
        raise HomeLBMError(f"{what}: {msg} (status {rc})")


def require_cuda(device=None):
    """The compute path is CUDA only; fail loudly otherwise."""
    import torch

    if not torch.cuda.is_available():
        raise HomeLBMError("openhomelbm_b200 needs a CUDA device (sm_100a); none is available")
    load()
    return torch.device(device if device is not None else "cuda")


def ptr(t):
    return None if t is None else c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)


DTYPES = {"float32": HL_F32, "float16": HL_F16, "bfloat16": HL_BF16, "float64": HL_F64}


def torch_dtype(code: int):
    import torch

    return {HL_F32: torch.float32, HL_F16: torch.float16, HL_BF16: torch.bfloat16, HL_F64: torch.float64}[code]


_TUNING: dict = {}


def set_tuning(key: str, value: int) -> None:
    """hl_set_tuning: process-wide kernel selection / work split knobs (see homelbm.h)."""
    check(lib().hl_set_tuning(key.encode(), int(value)), "hl_set_tuning")
    _TUNING[key] = int(value)


def get_tuning(key: str) -> int:
    """The value last set through set_tuning (0, the library's automatic choice, if never set)."""
    return _TUNING.get(key, 0)
