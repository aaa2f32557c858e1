"""Parity of the benchmarked kernel at the benchmark's own size: the D3Q27 Taylor-Green vortex,
periodic 256^3, float32 storage, u0 = 0.04, Re = 1600 (nu = u0 (256 / 2 pi) / 1600), 100 steps,
through LBM_Solver3D (the TMA-staged stream-collide kernel, the one bench.py times).

Criterion (oracle.oracle.check_parity): (a) relative L2 of rho, u and Pi/rho against the
binary32 oracle (bit-exact to the reference's stream_and_collide_3d,
envs/lbm3d/lbm_func_3d.py:364-604) within 1e-5 after 100 steps; (b) per field, the max error
against binary64 no larger than 3x the binary32 oracle's own. The binary64 side is the float64
storage build of the plain kernel on the GPU (the accuracy oracle): it evaluates the same
algorithm in binary64, so its distance from the CPU binary64 evaluation (~1e-15) is far below
the binary32 errors the criterion compares. The CPU oracle's 100 steps at 256^3 take one to a
few minutes on the host's threads.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N, U0, STEPS = 256, 0.04, 100


def _tgv(n, u0):
    x = 2 * np.pi * np.arange(n) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    ux = u0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    uy = -u0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    uz = np.zeros_like(ux)
    rho = 1 + 3 * (u0 ** 2 / 16) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2)
    return np.stack([rho, ux, uy, uz, ux * ux, uy * uy, uz * uz, ux * uy, ux * uz, uy * uz]).astype(np.float32)


def _gpu_run(storage, init, vis):
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    s = LBM_Solver3D(N, N, N, solid_num=1, periodic=True, storage=storage, with_flag=False, with_force=False)
    s.set_viscosity(vis)
    f = s.flows[0]
    t = torch.from_numpy(init).to(device=f.device, dtype=f.moments[0].dtype)
    f.moments[0].copy_(t)
    f.moments[1].copy_(t)
    del t
    for _ in range(STEPS):
        s.step()
    out = f.cur.cpu().numpy()
    del s, f
    torch.cuda.empty_cache()
    return out


def test_tgv_256_100_steps_tma_kernel_vs_oracle():
    from openhomelbm_b200 import _lib

    vis = U0 * (N / (2 * np.pi)) / 1600.0
    vis32 = float(np.float32(vis))
    init = _tgv(N, U0)
    _lib.set_tuning("d3q27_kernel", 0)  # automatic: the TMA kernel at this size, as in bench.py
    got = _gpu_run("float32", init, vis32)
    ref64 = _gpu_run("float64", init.astype(np.float64), vis32)
    assert np.isfinite(got).all() and np.isfinite(ref64).all()
    m, p = init.copy(), init.copy()
    for _ in range(STEPS):
        new, _ = orc.step_3d(m, p, vis_shear=np.float32(vis32), periodic=True, nthreads=0)
        m, p = new, m
    l2 = orc.rel_l2(got, m)
    own = orc.moment_errors(m, ref64)
    ours = orc.moment_errors(got, ref64)
    print(f"\n256^3 TGV, 100 steps: rel L2 vs binary32 oracle {l2}; max scaled error vs binary64: "
          f"kernel {ours.max():.3e}, binary32 oracle {own.max():.3e}")
    msgs = orc.check_parity(got, m, ref64)
    assert not msgs, msgs
