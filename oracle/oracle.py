"""ctypes binding of the CPU oracle (``liboracle.so``, built from ``homelbm_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg are the only callers. The product library never imports this module.

Each step function runs one ``LBM_Solver.step`` / ``LBM_Solver3D.step`` of one world of the
reference (envs/lbm/lbm_solver.py:104-141, envs/lbm3d/lbm_solver_3d.py:95-127) on NumPy
arrays, in binary32 (``dtype=np.float32``, the parity oracle) or binary64 (the accuracy
oracle), and returns the post-collision moments (the new current state after the swap).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (in place) and return the library path."""
    src = os.path.join(HERE, "homelbm_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# ----------------------------------------------------------------------------- 2D
@dataclass
class Solids2D:
    """Polygon solids of one 2D world (HomeFlow fields, envs/lbm/lbm_core.py:57-79)."""

    line: np.ndarray            # (n, max_seg, 2) local polygon vertices
    line_num: np.ndarray        # (n,) int32
    position: np.ndarray        # (n, 2)
    angle: np.ndarray           # (n,)
    scale: np.ndarray           # (n,)
    mass_center: np.ndarray     # (n, 2)
    max_radius: np.ndarray      # (n,)
    tf: Optional[np.ndarray] = None       # (n, max_seg, 2) solid_line_transformed
    tf_last: Optional[np.ndarray] = None  # (n, max_seg, 2) solid_line_transformed_last

    def cast(self, dt):
        for k in ("line", "position", "angle", "scale", "mass_center", "max_radius"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dt))
        self.line_num = np.ascontiguousarray(self.line_num, np.int32)
        if self.tf is None:
            self.tf = np.zeros_like(self.line)
            self.tf_last = np.zeros_like(self.line)
        self.tf = np.ascontiguousarray(self.tf, dt)
        self.tf_last = np.ascontiguousarray(self.tf_last, dt)
        return self


def step_2d(moments, post=None, *, vis_shear, bc_type, bc_value, flag=None, forcex=None, forcey=None,
            solids: Optional[Solids2D] = None, periodic=False, grid_length=None, time_step=1.0,
            dtype=np.float32, nthreads=1):
    """One D2Q9 step. ``moments`` is (6, nx, ny).

    ``post`` is the other buffer of the pair (the reference's ``*_post`` fields): its
    border cells are read by ``apply_bc`` before they are rewritten, so a faithful run
    passes the previous step's input here. Returns (new_moments, loads (n, 3)); the
    returned moments are ``post`` itself when it was given with the right dtype.
    """
    dt = np.dtype(dtype).type
    cur = np.ascontiguousarray(moments, dt)
    _, nx, ny = cur.shape
    post = cur.copy() if post is None else np.ascontiguousarray(post, dt)
    ct = ctypes.c_float if dt is np.float32 else ctypes.c_double
    if grid_length is None:
        grid_length = 1.0 / nx
    bct = np.ascontiguousarray(bc_type, np.int32)
    bcv = np.ascontiguousarray(bc_value, dt).reshape(4, 2)
    fl = None if flag is None else np.ascontiguousarray(flag, np.int32)
    fx = None if forcex is None else np.ascontiguousarray(forcex, dt)
    fy = None if forcey is None else np.ascontiguousarray(forcey, dt)
    if solids is not None:
        s = solids.cast(dt)
        n_obj, max_seg = s.line.shape[0], s.line.shape[1]
    else:
        s, n_obj, max_seg = None, 0, 1
    loads = np.zeros((max(n_obj, 1), 3), dt)
    fn = lib().oracle_step_2d_f32 if dt is np.float32 else lib().oracle_step_2d_f64
    rc = fn(ctypes.c_int(nx), ctypes.c_int(ny), ct(vis_shear), ct(grid_length), ct(time_step),
            _p(bct), _p(bcv), ctypes.c_int(int(periodic)), _p(cur), _p(post), _p(fl), _p(fx), _p(fy),
            ctypes.c_int(n_obj), ctypes.c_int(max_seg),
            _p(s.line if s else None), _p(s.line_num if s else None), _p(s.tf if s else None),
            _p(s.tf_last if s else None), _p(s.position if s else None), _p(s.angle if s else None),
            _p(s.scale if s else None), _p(s.mass_center if s else None),
            _p(s.max_radius if s else None), _p(loads), ctypes.c_int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle_step_2d failed: {rc}")
    return post, loads[:n_obj]


# ----------------------------------------------------------------------------- 3D
@dataclass
class Solids3D:
    """Triangle-mesh solids of one 3D world (HomeFlow3D fields, lbm_core_3d.py:91-119)."""

    tri_offset: np.ndarray      # (n+1,) int32 offsets into tris
    tris: np.ndarray            # (total, 3, 3) body-local, scaled vertices
    transforms: np.ndarray      # (n, 7) p, q(xyzw)
    transforms_last: np.ndarray  # (n, 7)
    initialized: np.ndarray     # (n,) int32
    position: np.ndarray        # (n, 3)
    bound_radius: np.ndarray    # (n,)
    scale_sizes: Optional[np.ndarray] = None  # (n, 3), ones by default
    linear_v: Optional[np.ndarray] = None     # (n, 3)
    angle_v: Optional[np.ndarray] = None      # (n, 3)

    def cast(self, dt):
        n = len(self.tri_offset) - 1
        if self.scale_sizes is None:
            self.scale_sizes = np.ones((n, 3))
        if self.linear_v is None:
            self.linear_v = np.zeros((n, 3))
        if self.angle_v is None:
            self.angle_v = np.zeros((n, 3))
        for k in ("tris", "transforms", "transforms_last", "position", "bound_radius",
                  "scale_sizes", "linear_v", "angle_v"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dt))
        self.tri_offset = np.ascontiguousarray(self.tri_offset, np.int32)
        self.initialized = np.ascontiguousarray(self.initialized, np.int32)
        return self


def step_3d(moments, post=None, *, vis_shear, bc_type=(1,) * 6, bc_value=((0, 0, 0),) * 6, flag=None,
            force=None, solids: Optional[Solids3D] = None, periodic=False, dtype=np.float32,
            nthreads=1):
    """One D3Q27 step. ``moments`` is (10, nx, ny, nz); ``post`` as in :func:`step_2d`.

    Returns (new_moments, loads (n, 6)).
    """
    dt = np.dtype(dtype).type
    cur = np.ascontiguousarray(moments, dt)
    _, nx, ny, nz = cur.shape
    post = cur.copy() if post is None else np.ascontiguousarray(post, dt)
    ct = ctypes.c_float if dt is np.float32 else ctypes.c_double
    bct = np.ascontiguousarray(bc_type, np.int32)
    bcv = np.ascontiguousarray(bc_value, dt).reshape(6, 3)
    fl = None if flag is None else np.ascontiguousarray(flag, np.int32)
    fo = None if force is None else np.ascontiguousarray(force, dt)
    if solids is not None:
        s = solids.cast(dt)
        n_obj = len(s.tri_offset) - 1
    else:
        s, n_obj = None, 0
    zero_off = np.zeros(1, np.int32)
    loads = np.zeros((max(n_obj, 1), 6), dt)
    fn = lib().oracle_step_3d_f32 if dt is np.float32 else lib().oracle_step_3d_f64
    rc = fn(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(nz), ct(vis_shear), _p(bct), _p(bcv),
            ctypes.c_int(int(periodic)), _p(cur), _p(post), _p(fl), _p(fo), ctypes.c_int(n_obj),
            _p(s.tri_offset if s else zero_off), _p(s.tris if s else None),
            _p(s.transforms if s else None), _p(s.transforms_last if s else None),
            _p(s.initialized if s else None), _p(s.scale_sizes if s else None),
            _p(s.position if s else None), _p(s.bound_radius if s else None),
            _p(s.linear_v if s else None), _p(s.angle_v if s else None), _p(loads),
            ctypes.c_int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle_step_3d failed: {rc}")
    return post, loads[:n_obj]


def border_flags_2d(nx, ny):
    """InitBoundary (envs/lbm/lbm_func.py:17-23) on an all-fluid grid."""
    f = np.zeros((nx, ny), np.int32)
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = 2
    return f


def border_flags_3d(nx, ny, nz):
    """InitBoundary3D (envs/lbm3d/lbm_func_3d.py:13-19)."""
    f = np.zeros((nx, ny, nz), np.int32)
    f[0], f[-1], f[:, 0], f[:, -1], f[:, :, 0], f[:, :, -1] = 2, 2, 2, 2, 2, 2
    return f


def moment_errors(got, ref):
    """Per-field errors of D2Q9 (6 planes) or D3Q27 (10 planes) moments, each divided by the
    scale of the quantity it stores:

    * rho by max|rho|;
    * every velocity component by the largest speed component of the field (max |u_a| over a);
    * a diagonal S_aa by max|S_aa + 1/3|: the reference stores S_aa = Pi_aa/rho - 1/3 and that
      subtraction leaves about one binary32 ulp of 1/3 (3e-8) of absolute noise in S_aa, so
      S_aa is only defined to that precision relative to Pi_aa/rho;
    * an off-diagonal S_ab by the largest off-diagonal magnitude of the field.
    """
    import numpy as np

    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    nm = ref.shape[0]
    if nm == 6:
        vel, diag, off = [1, 2], [3, 4], [5]
    elif nm == 10:
        vel, diag, off = [1, 2, 3], [4, 5, 6], [7, 8, 9]
    else:
        raise ValueError(nm)
    d = np.abs(got - ref)
    out = np.zeros(nm)
    out[0] = d[0].max() / np.abs(ref[0]).max()
    us = max(np.abs(ref[vel]).max(), 1e-12)
    for k in vel:
        out[k] = d[k].max() / us
    for k in diag:
        out[k] = d[k].max() / np.abs(ref[k] + 1.0 / 3.0).max()
    os_ = max(np.abs(ref[off]).max(), 1e-12)
    for k in off:
        out[k] = d[k].max() / os_
    return out


def rel_l2(got, ref):
    """Relative L2 errors of the moment groups: rho, the velocity vector and the second-moment
    tensor Pi/rho = S + I/3 (the quantity the reference's S is taken from)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    nm = ref.shape[0]
    nd = 2 if nm == 6 else 3
    vel = slice(1, 1 + nd)
    sec = slice(1 + nd, nm)
    shift = np.zeros_like(ref[sec])
    shift[:nd] = 1.0 / 3.0
    return {
        "rho": float(np.linalg.norm(got[0] - ref[0]) / np.linalg.norm(ref[0])),
        "u": float(np.linalg.norm(got[vel] - ref[vel]) / max(np.linalg.norm(ref[vel]), 1e-300)),
        "Pi": float(np.linalg.norm(got[sec] - ref[sec]) / np.linalg.norm(ref[sec] + shift)),
    }


def check_parity(got, ref32, ref64, tol=1e-5, factor=3.0, floor=1e-7):
    """The parity criterion of the tests.

    (a) relative L2 of rho, u and Pi/rho against the binary32 reference (the oracle, which is
        bit-exact to the reference's kernels) within ``tol``;
    (b) per field, the max error against the binary64 evaluation of the same algorithm no
        larger than ``factor`` times the reference's own binary32 error (plus ``floor``): the
        CUDA result is as accurate as the reference. One binary32-vs-binary64 comparison is a
        noisy estimate of a noise floor (moving walls, for instance, take their velocity from
        differences of binary32 absolute positions), hence the factor of 3.
    Returns a description of the failures (empty when both hold).
    """
    msgs = []
    l2 = rel_l2(got, ref32)
    bad = {k: v for k, v in l2.items() if not v <= tol}
    if bad:
        msgs.append(f"relative L2 vs reference above {tol}: {bad}")
    e_got = moment_errors(got, ref64)
    e_ref = moment_errors(ref32, ref64)
    over = np.nonzero(~(e_got <= factor * e_ref + floor))[0]
    if len(over):
        msgs.append("less accurate than the reference on planes " +
                    ", ".join(f"{k}: {e_got[k]:.2e} > {factor}x{e_ref[k]:.2e}" for k in over))
    return msgs
