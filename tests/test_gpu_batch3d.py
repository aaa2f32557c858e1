"""Batched D3Q27 stream-collide (hl_d3q27_stream_collide_batch) on the GPU.

The per-cell arithmetic of the TMA kernel does not depend on how x is split into chunks or
which CTA takes an item, so one launch over several domains must write, in every domain,
exactly what a launch per domain writes. The served engine built on it must give the same
loads and fields as the engine that runs each domain's control step as its own graph (loads
to 1e-6 of their magnitude: their binary64 sums are atomics in varying order).
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solver(nx, ny, nz, storage, seed):
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    s = LBM_Solver3D(nx, ny, nz, storage=storage, use_graph=False, with_flag=False, with_force=False,
                     **({} if storage == "float32" else dict(u_scale=0.05, s_scale=2e-3)))
    s.set_viscosity(0.02)
    s.set_uniform_flow(0.02, -0.01, 0.005)
    f = s.flows[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    for m in f.moments:  # a non-uniform state: small seeded noise on every stored moment
        noise = (torch.rand(m.shape, generator=g) - 0.5) * (2e-3 if storage == "float32" else 0.04)
        m.copy_((m.float() + noise.to(m.device)).to(m.dtype))
    return s


@pytest.mark.parametrize("storage", ["float32", "float16", "bfloat16"])
def test_batched_stream_collide_equals_one_launch_per_domain(storage):
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.serving import BatchStep

    class D:  # the part of a served domain BatchStep reads
        def __init__(self, solver):
            self.solver = solver
            self.req = type("R", (), {"substeps": 2})()

    sizes = [(64, 64, 64), (96, 48, 64), (40, 32, 96), (128, 96, 128)]
    solvers = [_solver(*sz, storage, seed=k) for k, sz in enumerate(sizes)]
    st = torch.cuda.current_stream()
    batch = BatchStep([D(s) for s in solvers], st)
    assert batch.n == 4 and batch.n_items > 0
    L = _lib.lib()
    for parity in (0, 1):
        ref = []
        for s in solvers:
            f = s.flows[0]
            f.moments[parity ^ 1].zero_()
            _lib.check(L.hl_d3q27_stream_collide(f.world_struct(parity), float(f.vis_shear), None, _lib.stream_ptr()),
                       "per domain")
            ref.append(f.moments[parity ^ 1].clone())
        for s in solvers:
            s.flows[0].moments[parity ^ 1].fill_(7)
        batch.launch(parity, st)
        torch.cuda.synchronize()
        assert int(batch.status.item()) == 0
        for s, r in zip(solvers, ref):
            out = s.flows[0].moments[parity ^ 1]
            assert torch.equal(out[:, 1:-1, 1:-1, 1:-1], r[:, 1:-1, 1:-1, 1:-1]), (s.nx, s.ny, s.nz, parity)
            for face in (out[:, 0], out[:, -1], out[:, :, 0], out[:, :, -1], out[:, :, :, 0], out[:, :, :, -1]):
                assert bool((face == 7).all())  # wall cells are the boundary pass's


def test_served_engine_batched_equals_per_domain_graphs():
    from openhomelbm_b200.serving import Request, ServeEngine

    # with 6 control steps the set of three holds long enough for the engine to capture and
    # replay its tick graph; the set changes (a request finishes, another is admitted) run eagerly
    reqs = [Request(0, 64, 11, 0.0, control_steps=6, substeps=4), Request(1, 96, 12, 0.0, control_steps=7, substeps=4),
            Request(2, 64, 13, 0.0, control_steps=2, substeps=4), Request(3, 128, 14, 0.0, control_steps=6, substeps=4)]
    a = ServeEngine(storage="float16", max_active=3, batched=True, keep_fields=True).run(reqs, realtime=False)
    b = ServeEngine(storage="float16", max_active=3, batched=False, keep_fields=True).run(reqs, realtime=False)
    assert a.max_active == 3 and set(a.results) == {0, 1, 2, 3}
    for r in reqs:
        x, y = a.results[r.rid].astype(np.float64), b.results[r.rid].astype(np.float64)
        assert np.abs(y).max() > 0
        assert np.abs(x - y).max() <= 1e-6 * np.abs(y).max(), r.rid
        np.testing.assert_array_equal(a.fields[r.rid], b.fields[r.rid])


def test_batch_rejects_bad_arguments():
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.lbm3d import LBM_Solver3D
    from openhomelbm_b200.serving import Domain, Request

    L = _lib.lib()
    s = LBM_Solver3D(32, 32, 32, periodic=True, use_graph=False)
    worlds = (_lib.hl_world3d * 1)(s.flows[0].world_struct(0))
    buf = torch.empty(int(L.hl_d3q27_batch_bytes(1)) + 64, dtype=torch.uint8, device="cuda")
    ptr = (buf.data_ptr() + 63) // 64 * 64
    n = ctypes.c_int(0)
    with pytest.raises(ValueError):  # periodic
        _lib.check(L.hl_d3q27_batch_prepare(worlds, 1, ptr, buf.numel() - 64, ctypes.byref(n), _lib.stream_ptr()))
    w = _solver(32, 32, 32, "float32", 0).flows[0].world_struct(0)
    worlds = (_lib.hl_world3d * 1)(w)
    with pytest.raises(ValueError):  # misaligned descriptors
        _lib.check(L.hl_d3q27_batch_prepare(worlds, 1, ptr + 16, buf.numel() - 64, ctypes.byref(n), _lib.stream_ptr()))
    _lib.check(L.hl_d3q27_batch_prepare(worlds, 1, ptr, buf.numel() - 64, ctypes.byref(n), _lib.stream_ptr()))
    assert n.value > 0
    with pytest.raises(ValueError):  # counts that were not prepared
        _lib.check(L.hl_d3q27_stream_collide_batch(ptr, 1, n.value + 1, 0.02, ctypes.byref(w.storage), 0, None,
                                                   _lib.stream_ptr()))
    with pytest.raises(ValueError):
        Domain(Request(0, 64, 1, 0.0, control_steps=1, substeps=3), "float16", 0.01, torch.device("cuda:0"))


@pytest.mark.parametrize("storage", ["float16", "float32", "bfloat16"])
def test_batched_cut_links_equal_per_domain(storage):
    """hl_d3q27_solid_links_batch over three served domains computes, between the same
    stream-collide and boundary launches, exactly the moments the per-domain cut links compute;
    the loads agree to binary32 rounding (binary64 sums in another order)."""
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.serving import Domain, LinkBatch, Request

    doms = [Domain(Request(k, side, 31 + k, 0.0, control_steps=4, substeps=2), storage, 0.01,
                   torch.device("cuda:0"), use_graph=False) for k, side in enumerate((64, 96, 128))]
    for step in range(2):  # swimmers moving, a developed flow
        for d in doms:
            d.stage_poses(step)
            d.launch()
        for d in doms:
            d.event.synchronize()
            d.finish(0.0)
    L = _lib.lib()
    st = _lib.stream_ptr()
    links = LinkBatch(doms, torch.cuda.current_stream())
    ref = []
    for d in doms:
        f = d.solver.flows[0]
        f.moments[1].zero_()
        d.solver._launch(0, st, loads_out=d._loads_out(0))
        torch.cuda.synchronize()
        ref.append((f.moments[1].clone(), d.loads_dev[0].clone()))
    for d in doms:
        f = d.solver.flows[0]
        f.moments[1].zero_()
        d.loads_dev.zero_()
        _lib.check(L.hl_d3q27_stream_collide(f.world_struct(0), float(f.vis_shear), None, st), "stream-collide")
    links.launch(0, torch.cuda.current_stream())
    for d in doms:
        d.solver._launch(0, st, stream_collide=False, solid_links=False)
    torch.cuda.synchronize()
    for d, (m, loads) in zip(doms, ref):
        assert torch.equal(d.solver.flows[0].moments[1], m), d.req.side
        a, b = d.loads_dev[0].double(), loads.double()
        assert b.abs().max() > 0
        assert (a - b).abs().max() <= 1e-6 * b.abs().max(), d.req.side


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_batched_boundaries_equal_per_domain(storage):
    """hl_d3q27_apply_bc_batch (three launches over all domains) writes, at both parities,
    exactly what hl_d3q27_apply_bc writes per domain: worlds of different shapes (odd sides
    included), random moments, a random boundary type per face (fixed velocity, zero gradient,
    or a type that keeps the cell's own velocity)."""
    from openhomelbm_b200 import _lib

    L = _lib.lib()
    st = _lib.stream_ptr()
    code = _lib.DTYPES[storage]
    sto = _lib.hl_storage(code, 0.05, 2e-3) if storage != "float32" else _lib.hl_storage(code, 1.0, 1.0)
    rng = np.random.default_rng(5)
    shapes = [(16, 24, 32), (33, 17, 20), (8, 9, 10), (40, 32, 32), (3, 5, 7)]
    doms = []
    for nx, ny, nz in shapes:
        b0 = torch.tensor(rng.uniform(-0.5, 0.5, (10, nx, ny, nz)), dtype=_lib.torch_dtype(code), device="cuda")
        b1 = torch.tensor(rng.uniform(-0.5, 0.5, (10, nx, ny, nz)), dtype=_lib.torch_dtype(code), device="cuda")
        if storage == "float32":  # rho near 1
            b0[0] += 1.0
            b1[0] += 1.0
        bc = _lib.hl_bc3d()
        for f in range(6):
            bc.bc_type[f] = int(rng.integers(0, 3))
            for k in range(3):
                bc.bc_value[f][k] = float(rng.uniform(-0.03, 0.03))
        w = _lib.hl_world3d(nx, ny, nz, sto, b0.data_ptr(), b1.data_ptr(), None, None, 0)
        scratch = torch.zeros(int(L.hl_d3q27_bc_scratch_bytes(ctypes.byref(w))), dtype=torch.uint8, device="cuda")
        doms.append(dict(b=(b0, b1), bc=bc, shape=(nx, ny, nz), scratch=scratch))
    n = len(doms)
    nbytes = int(L.hl_d3q27_bc_batch_bytes(n))
    desc = torch.empty(nbytes + 16, dtype=torch.uint8, device="cuda")
    ptr = (desc.data_ptr() + 15) // 16 * 16
    worlds = (_lib.hl_world3d * n)(*[_lib.hl_world3d(*d["shape"], sto, d["b"][0].data_ptr(), d["b"][1].data_ptr(),
                                                     None, None, 0) for d in doms])
    bcs = (_lib.hl_bc3d * n)(*[d["bc"] for d in doms])
    scr = (ctypes.c_void_p * n)(*[d["scratch"].data_ptr() for d in doms])
    _lib.check(L.hl_d3q27_bc_batch_prepare(worlds, bcs, scr, n, ptr, nbytes, st), "prepare")
    for parity in (0, 1):
        start = [d["b"][1 - parity].clone() for d in doms]  # the buffer the pass writes
        ref = []
        for d, s0 in zip(doms, start):
            out = d["b"][1 - parity]
            out.copy_(s0)
            cur = d["b"][parity]
            w = _lib.hl_world3d(*d["shape"], sto, cur.data_ptr(), out.data_ptr(), None, None, 0)
            _lib.check(L.hl_d3q27_apply_bc(ctypes.byref(w), ctypes.byref(d["bc"]), d["scratch"].data_ptr(), st), "bc")
            torch.cuda.synchronize()
            ref.append(out.clone())
            assert not torch.equal(out, s0)  # the pass changed the border
            out.copy_(s0)
        _lib.check(L.hl_d3q27_apply_bc_batch(ptr, n, parity, st), "batched bc")
        torch.cuda.synchronize()
        for d, r in zip(doms, ref):
            assert torch.equal(d["b"][1 - parity], r), (d["shape"], parity)
    with pytest.raises(ValueError):  # counts that were not prepared
        _lib.check(L.hl_d3q27_apply_bc_batch(ptr, n + 1, 0, st))
    with pytest.raises(ValueError):  # a periodic world
        pw = (_lib.hl_world3d * 1)(_lib.hl_world3d(8, 8, 8, sto, doms[2]["b"][0].data_ptr(),
                                                   doms[2]["b"][1].data_ptr(), None, None, 1))
        _lib.check(L.hl_d3q27_bc_batch_prepare(pw, bcs, scr, 1, ptr, nbytes, st))
