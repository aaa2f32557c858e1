"""hl_d3q27_stream_collide_noalloc: the D3Q27 stream-collide with mass / health diagnostics for
callers that cannot allocate device memory (a host whose HBM is fully reserved by its own
caching allocator or by resident domains, a control loop that must not pay allocation latency).

The entry point keeps its scratch in a fixed-size array inside the library instead of a
caller-provided buffer. These tests call it through the C ABI and check each of two calls in
a row against hl_d3q27_stream_collide given its own zeroed scratch buffer: the moments within
the parity tests' tolerance of 1e-5 on their scaled errors (conftest.moment_errors: each field's
max error over the scale of the quantity it stores; the two entry points may use different
kernels, which round differently), the mass within 1e-9 relative and the health count exactly,
and the mass and health against their definitions evaluated on the written field.
The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import moment_errors
from openhomelbm_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _world(shape, dtype_code, cur, post, periodic, flag=None, force=None):
    nx, ny, nz = shape
    return _lib.hl_world3d(nx, ny, nz, _lib.hl_storage(dtype_code, 1.0, 1.0), cur.data_ptr(), post.data_ptr(),
                           None if flag is None else flag.data_ptr(), None if force is None else force.data_ptr(),
                           int(periodic))


def _setup(shape, storage, periodic, poison):
    _lib.require_cuda()
    lib = _lib.lib()
    code = _lib.DTYPES[storage]
    dt = _lib.torch_dtype(code)
    nx, ny, nz = shape
    st = _lib.stream_ptr()
    a = torch.zeros((10, nx, ny, nz), dtype=dt, device="cuda")
    b = torch.zeros_like(a)
    flag = None
    force = None
    if periodic:
        _lib.check(lib.hl_d3q27_init_tgv(nx, ny, nz, _lib.hl_storage(code, 1.0, 1.0), a.data_ptr(), b.data_ptr(),
                                         0.05, st), "init_tgv")
    else:
        force = torch.zeros((3, nx, ny, nz), dtype=torch.float32, device="cuda")
        _lib.check(lib.hl_d3q27_init_uniform(nx, ny, nz, _lib.hl_storage(code, 1.0, 1.0), a.data_ptr(),
                                             b.data_ptr(), force.data_ptr(), 0.02, -0.01, 0.03, st), "init_uniform")
        flag = torch.zeros((nx, ny, nz), dtype=torch.int32, device="cuda")
        _lib.check(lib.hl_d3q27_init_boundary(nx, ny, nz, flag.data_ptr(), st), "init_boundary")
        force[0].fill_(1e-5)
    if poison:
        # a non-finite cell: the clamp of the rebuilt populations decides what it becomes
        a[0, nx // 2, ny // 3, nz // 4] = float("inf")
        a[1, 3, 5, 7] = float("nan")
    torch.cuda.synchronize()
    return lib, code, a, b, flag, force


@pytest.mark.parametrize("shape,storage,periodic,poison", [
    ((32, 32, 32), "float32", True, False),
    ((24, 20, 18), "float32", False, False),
    ((16, 16, 32), "float64", True, False),
    ((24, 16, 32), "float32", True, True),
])
def test_noalloc_matches_allocating_entry_point(shape, storage, periodic, poison):
    lib, code, a, b, flag, force = _setup(shape, storage, periodic, poison)
    # Non-finite values take the same path only through the same kernel: the poisoned case
    # pins the allocating entry point to the kernel the allocation-free one uses.
    _lib.set_tuning("d3q27_kernel", 1 if poison else 0)
    try:
        _run_pair(lib, code, a, b, flag, force, shape, periodic, poison)
    finally:
        _lib.set_tuning("d3q27_kernel", 0)


def _run_pair(lib, code, a, b, flag, force, shape, periodic, poison):
    a2, b2 = a.clone(), b.clone()
    st = _lib.stream_ptr()
    vis = 0.01

    # existing entry point, with scratch allocated by the caller
    w = _world(shape, code, a, b, periodic, flag, force)
    nbytes = lib.hl_d3q27_scratch_bytes(ctypes.byref(w))
    scratch = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    bad = torch.zeros(2, dtype=torch.int32, device="cuda")
    # allocation-free entry point
    out2 = torch.zeros(2, dtype=torch.float64, device="cuda")
    bad2 = torch.zeros(2, dtype=torch.int32, device="cuda")

    bufs, bufs2 = (a, b), (a2, b2)
    for call in range(2):
        src, dst = bufs[call % 2], bufs[(call + 1) % 2]
        src2, dst2 = bufs2[call % 2], bufs2[(call + 1) % 2]
        w = _world(shape, code, src, dst, periodic, flag, force)
        d = _lib.hl_diag(scratch.data_ptr(), nbytes, out[call:].data_ptr(), bad[call:].data_ptr())
        _lib.check(lib.hl_d3q27_stream_collide(ctypes.byref(w), vis, ctypes.byref(d), st), "stream_collide")
        w2 = _world(shape, code, src2, dst2, periodic, flag, force)
        _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(w2), vis, out2[call:].data_ptr(),
                                                       bad2[call:].data_ptr(), st), "stream_collide_noalloc")
        torch.cuda.synchronize()

        ref = dst.double().cpu().numpy()
        got = dst2.double().cpu().numpy()
        if poison:
            ok = np.isfinite(ref).all(axis=0)
            assert (np.isfinite(got).all(axis=0) == ok).all(), call
            ref, got = ref[:, ok], got[:, ok]
        errs = moment_errors(got, ref)
        assert errs.max() <= TOL, (call, errs)
        m, m2 = out[call].item(), out2[call].item()
        assert _close(m2, m), (call, m, m2)
        assert bad2[call].item() == bad[call].item(), (call, bad[call].item(), bad2[call].item())
        # and both are what the output field says
        mass, health = _expected_diag(dst2, flag)
        assert _close(m2, mass), (call, m2, mass)
        assert bad2[call].item() == health, (call, bad2[call].item(), health)


def _close(x, y):
    if not (np.isfinite(x) and np.isfinite(y)):
        return not np.isfinite(x) and not np.isfinite(y)
    return abs(x - y) <= 1e-9 * abs(y)


def _expected_diag(field, flag):
    """Mass (sum of rho) and health (cells with a non-finite moment or rho <= 0) over the
    updated cells of a written field: every cell of a periodic world, else ML_FLUID cells."""
    f = field.double().cpu().numpy()
    upd = np.ones(f.shape[1:], bool) if flag is None else (flag.cpu().numpy() == 0)
    bad = ~(np.isfinite(f).all(axis=0) & (f[0] > 0))
    return float(f[0][upd].sum()), int((bad & upd).sum())


def test_noalloc_optional_outputs_and_rejections():
    lib, code, a, b, flag, force = _setup((16, 16, 32), "float32", True, False)
    st = _lib.stream_ptr()
    w = _world((16, 16, 32), code, a, b, True)
    # mass and health may be NULL: the step itself still runs
    _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(w), 0.01, None, None, st), "noalloc")
    torch.cuda.synchronize()
    assert torch.isfinite(b).all()
    # reduced-precision storages are not served by this entry point
    h = torch.zeros((10, 16, 16, 32), dtype=torch.float16, device="cuda")
    h2 = torch.zeros_like(h)
    wh = _world((16, 16, 32), _lib.HL_F16, h, h2, True)
    rc = lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(wh), 0.01, None, None, st)
    assert rc == _lib.HL_ERR_ARG
    assert b"float32 or float64" in lib.hl_last_error()


def test_noalloc_back_to_back_on_one_stream():
    """Two calls queued on one stream with no host synchronisation between them share the one
    scratch array safely (stream order serialises them); each call's mass and health match the
    definitions on the field that call wrote."""
    shape = (24, 16, 32)
    lib, code, a, b, flag, force = _setup(shape, "float32", True, False)
    c = torch.empty_like(a)
    st = _lib.stream_ptr()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    bad = torch.full((2,), -1, dtype=torch.int32, device="cuda")
    w1 = _world(shape, code, a, b, True)
    w2 = _world(shape, code, b, c, True)
    _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(w1), 0.01, out[0:].data_ptr(), bad[0:].data_ptr(),
                                                   st), "noalloc 1")
    _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(w2), 0.01, out[1:].data_ptr(), bad[1:].data_ptr(),
                                                   st), "noalloc 2")
    torch.cuda.synchronize()
    for k, field in enumerate((b, c)):
        mass, health = _expected_diag(field, None)
        assert _close(out[k].item(), mass), (k, out[k].item(), mass)
        assert bad[k].item() == health == 0, (k, bad[k].item(), health)
    assert out[0].item() != 0.0 and out[1].item() != 0.0


def test_noalloc_captured_in_a_graph_after_a_first_call():
    """The documented order: a first call outside any capture resolves the array's address;
    a later call may then be captured in a CUDA graph. Each replay writes the same field, mass
    and health as a direct call on the same input."""
    shape = (24, 16, 32)
    lib, code, a, b, flag, force = _setup(shape, "float32", True, False)
    c = torch.empty_like(a)
    direct = torch.empty_like(a)
    st = _lib.stream_ptr()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    bad = torch.full((3,), -1, dtype=torch.int32, device="cuda")
    # first call, uncaptured: a -> b
    _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(_world(shape, code, a, b, True)), 0.01,
                                                   out[0:].data_ptr(), bad[0:].data_ptr(), st), "noalloc 1")
    # the reference second step, uncaptured: b -> direct
    _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(_world(shape, code, b, direct, True)), 0.01,
                                                   out[1:].data_ptr(), bad[1:].data_ptr(), st), "noalloc 2")
    torch.cuda.synchronize()
    w = _world(shape, code, b, c, True)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        _lib.check(lib.hl_d3q27_stream_collide_noalloc(ctypes.byref(w), 0.01, out[2:].data_ptr(),
                                                       bad[2:].data_ptr(), _lib.stream_ptr()), "noalloc captured")
    for replay in range(2):
        c.fill_(float("nan"))
        out[2] = 0.0
        bad[2] = -1
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(c, direct), replay
        assert out[2].item() == out[1].item(), (replay, out[2].item(), out[1].item())
        assert bad[2].item() == bad[1].item() == 0, replay
    mass, health = _expected_diag(c, None)
    assert _close(out[2].item(), mass) and health == 0
    del g
