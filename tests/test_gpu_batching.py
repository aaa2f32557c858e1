"""Batching form on the GPU (openhomelbm_b200.batching, hl_d2q9_step_tiles).

* The persistent tile launch against the gridded stream phase of hl_d2q9_step_batch on uneven
  worlds (sizes that are no multiple of any tile, a periodic world, a forced world, capsule
  solids): identical post moments for every tile shape and grid, binary32 and float16.
* The tile path against the oracle on uneven worlds with moving capsules: the parity criterion
  of oracle.check_parity for the moments; the loads against the binary64 oracle within 3x the
  binary32 oracle's own error (plus 1e-5 of the largest load).
* The autotuner: every candidate timed, the fastest chosen, the choice cached.
* The swimmer batch: each world's loads the same alone and in the batch, and the float16 batch
  against the plain float32 solver one world at a time.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

WORLDS = [  # nx, ny, periodic, forced, capsules
    (37, 29, False, False, 1),
    (130, 70, False, True, 0),
    (64, 64, True, False, 0),
    (200, 41, False, False, 2),
]


def _raw_init(f, rng):
    """Random moments near rest in the world's raw storage layout."""
    nx, ny = f.nx, f.ny
    rho = 1.0 + 1e-3 * rng.standard_normal((nx, ny))
    ux = 0.02 * rng.standard_normal((nx, ny))
    uy = 0.02 * rng.standard_normal((nx, ny))
    sn = 1e-4 * rng.standard_normal((3, nx, ny))
    if f.encoded:
        raw = np.stack([rho - 1.0, ux / f.u_scale, uy / f.u_scale, sn[0] / f.s_scale, sn[1] / f.s_scale,
                        sn[2] / f.s_scale])
    else:
        raw = np.stack([rho, ux, uy, ux * ux + sn[0], uy * uy + sn[1], ux * uy + sn[2]])
    t = torch.tensor(raw, dtype=f.moments[0].dtype, device=f.device)
    f.moments[0].copy_(t)
    f.moments[1].copy_(t)


def _make_worlds(storage, seed=3):
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.batching import capsule_polygon
    from openhomelbm_b200.lbm.lbm_core import HomeFlow

    rng = np.random.default_rng(seed)
    flows = []
    for nx, ny, periodic, forced, caps in WORLDS:
        f = HomeFlow()
        f.Initialize(nx, ny, n_objects=2, storage=storage, u_scale=0.05, s_scale=1e-3, periodic=periodic)
        f.vis_shear = 0.02
        f.bc_type = [0, 1, 1, 1]
        f.bc_value = np.array([[0.03, 0.0], [0, 0], [0, 0], [0, 0]], np.float32)
        if not periodic:
            _lib.check(_lib.lib().hl_d2q9_init_boundary(nx, ny, _lib.ptr(f.flag), _lib.stream_ptr()), "flags")
        _raw_init(f, rng)
        if forced:
            f.force.copy_(torch.tensor(1e-5 * rng.standard_normal((2, nx, ny)), dtype=torch.float32, device=f.device))
            f.use_force = True
        for k in range(caps):
            f.configure_solid(k, capsule_polygon(4.0, 4.0), (0.3 * nx + 12 * k, 0.5 * ny + 0.3), angle=0.2 * k + 0.1,
                              scale=1.0 / nx)
        flows.append(f)
    return flows


def _segment_state(flows):
    return [(f.solid_line_transformed.clone(), f.solid_line_transformed_last.clone()) for f in flows]


def _restore(flows, seg, post0):
    for f, (a, b), p in zip(flows, seg, post0):
        f.solid_line_transformed.copy_(a)
        f.solid_line_transformed_last.copy_(b)
        f.moments[1].copy_(p)


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_tiles_identical_to_gridded_stream(storage):
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.batching import TileConfig, WorldBatch2D, tile_shapes

    flows = _make_worlds(storage)
    b = WorldBatch2D(flows)
    seg, post0 = _segment_state(flows), [f.moments[1].clone() for f in flows]
    L = _lib.lib()
    st = _lib.stream_ptr()
    _lib.check(L.hl_d2q9_step_batch(_lib.ptr(b.desc), b.n, 0, b.storage_code, max(f.nx for f in flows),
                                    max(f.ny for f in flows), int(b.any_solid), _lib.HL_PHASE_ALL, st), "gridded")
    ref = [f.moments[1].clone() for f in flows]
    ref_loads = [torch.stack([f.solid_forcex, f.solid_forcey, f.torque]).clone() for f in flows]
    assert b.any_solid
    for shape in tile_shapes():
        n_tiles = b.tiles(shape).shape[0]
        for ctas in (1, 7, n_tiles):
            _restore(flows, seg, post0)
            b.launch(0, st, TileConfig(shape[0], shape[1], ctas))
            torch.cuda.synchronize()
            for k, f in enumerate(flows):
                assert torch.equal(f.moments[1], ref[k]), (storage, shape, ctas, k)
                got = torch.stack([f.solid_forcex, f.solid_forcey, f.torque])
                torch.testing.assert_close(got, ref_loads[k], rtol=1e-6, atol=1e-12)


def test_tiles_match_oracle_with_moving_capsules():
    from openhomelbm_b200.batching import TileConfig, WorldBatch2D

    flows = _make_worlds("float32", seed=5)
    b = WorldBatch2D(flows)
    b.config = TileConfig(16, 32, 148)
    steps, v = 6, np.float32(0.01)
    init = [f.cur.cpu().numpy().astype(np.float64) for f in flows]
    states = []
    for f, m0 in zip(flows, init):
        n = f.n_objects
        # Solids2D.cast converts in place: one object per precision, each with its own segment state
        sol = lambda dt: orc.Solids2D(line=f.solid_line.cpu().numpy(), line_num=f.solid_line_num.cpu().numpy(),
                                      position=f.solid_position.cpu().numpy().astype(np.float64),
                                      angle=f.solid_angle.cpu().numpy().astype(np.float64),
                                      scale=f.solid_scale.cpu().numpy(),
                                      mass_center=f.solid_mass_center.cpu().numpy(),
                                      max_radius=f.solid_max_radius.cpu().numpy()).cast(dt)
        m32 = m0.astype(np.float32)
        states.append(dict(m32=m32, p32=m32.copy(), m64=m0.copy(), p64=m0.copy(), s32=sol(np.float32),
                           s64=sol(np.float64), n=n))
    for _ in range(steps):
        for f, s in zip(flows, states):
            if int(f.solid_line_num.max()) > 0:
                f.solid_position[:, 0] += float(v)
                for key in ("s32", "s64"):
                    s[key].position[:, 0] += s[key].position.dtype.type(v)
        b.upload()
        b.step()
        for f, s in zip(flows, states):
            kw = dict(vis_shear=np.float32(f.vis_shear), bc_type=f.bc_type, bc_value=f.bc_value,
                      flag=None if f.periodic else f.flag.cpu().numpy(), periodic=f.periodic,
                      forcex=f.force[0].cpu().numpy() if f.use_force else None,
                      forcey=f.force[1].cpu().numpy() if f.use_force else None, nthreads=0)
            has = int(f.solid_line_num.max()) > 0
            new32, loads32 = orc.step_2d(s["m32"], s["p32"], solids=s["s32"] if has else None, **kw)
            s["m32"], s["p32"] = new32, s["m32"]
            kw["vis_shear"] = float(np.float32(f.vis_shear))
            new64, loads64 = orc.step_2d(s["m64"], s["p64"], solids=s["s64"] if has else None, dtype=np.float64,
                                         **kw)
            s["m64"], s["p64"] = new64, s["m64"]
            s["loads32"], s["loads64"] = loads32, loads64
    for k, (f, s) in enumerate(zip(flows, states)):
        msgs = orc.check_parity(f.cur.cpu().numpy(), s["m32"], s["m64"])
        assert not msgs, (k, msgs)
        if int(f.solid_line_num.max()) > 0:
            # loads as accurate as the reference's binary32 arithmetic: against the binary64
            # evaluation, within 3x the binary32 reference's own error (+ 1e-5 of the largest)
            got = torch.stack([f.solid_forcex, f.solid_forcey, f.torque], 1).cpu().numpy().astype(np.float64)
            r32 = np.asarray(s["loads32"], np.float64)[: got.shape[0]]
            r64 = np.asarray(s["loads64"], np.float64)[: got.shape[0]]
            err, own = np.abs(got - r64).max(), np.abs(r32 - r64).max()
            assert err <= 3 * own + 1e-5 * np.abs(r64).max(), (k, err, own, got, r64)


def test_autotuner_times_every_candidate_and_caches():
    from openhomelbm_b200.batching import TileAutotuner, WorldBatch2D

    flows = _make_worlds("float16")
    b = WorldBatch2D(flows)
    tuner = TileAutotuner(ctas_per_sm=(1, 2), reps=2, warmup=1)
    before = [f.cur.clone() for f in flows]
    cfg = tuner.tune(b)
    table = tuner.table[b.signature()]
    assert set(table) == set(tuner.candidates(b))
    assert cfg == min(table, key=table.get) and b.config == cfg
    assert all(torch.equal(f.cur, x) for f, x in zip(flows, before))  # tuning leaves the state alone
    assert tuner.tune(b) is cfg


def _small_specs():
    from openhomelbm_b200.batching import CapsuleChain, SwimmerSpec

    sizes = [(200, 100), (256, 130), (180, 140)]
    return [SwimmerSpec(nx, ny, CapsuleChain(head=(0.25 * nx, 0.5 * ny), freq=0.004 + 0.002 * k))
            for k, (nx, ny) in enumerate(sizes)]


def test_swimmer_batch_same_alone_and_against_plain():
    from openhomelbm_b200.batching import SwimmerBatch2D, run_sequential_plain

    specs = _small_specs()
    steps = 3
    mix = SwimmerBatch2D(specs).run(steps)
    assert mix.loads.shape == (steps, 8, len(specs), 3, 8)
    assert np.isfinite(mix.loads).all() and np.abs(mix.loads).max() > 0
    alone = SwimmerBatch2D(specs[1:2]).run(steps)
    np.testing.assert_allclose(mix.loads[:, :, 1], alone.loads[:, :, 0], rtol=1e-5, atol=1e-9)
    plain = run_sequential_plain(specs, steps)
    a, p = mix.loads.astype(np.float64), plain.loads.astype(np.float64)
    rel = np.linalg.norm(a - p) / np.linalg.norm(p)
    assert rel < 2e-2, rel
