"""The D2Q9 Karman configuration (512 x 128, 96-gon cylinder of radius 12, Re = 100) on the
GPU against the oracle (tests/golden/make_cfg1.py; the oracle reproduces the reference's
kernels bit for bit on the golden cases):

* the moments after 100 steps within the parity criterion (oracle.check_parity), its L2 bound
  raised to 3x the reference's own binary32-vs-binary64 L2 difference where that exceeds 1e-5:
  in this impulsively started flow the clamped cut-link populations behind the cylinder
  amplify rounding, and the reference's binary32 result itself differs from binary64 by
  8e-4 (u) and 3e-3 (S) after 100 steps, so no implementation that rounds differently from
  the reference can stay within 1e-5 of it;
* drag and lift (solid_forcex, solid_forcey) after every one of 2000 steps: the means within
  1 % (lift: 1 % of the mean drag, the lift being noise-level before shedding starts), and
  every value within 3x the reference's own binary32 deviation from binary64.

The Strouhal number needs the shedding cycle, which this configuration reaches after about
40000 steps; bench.py --workload karman compares it over steps 70000-100000.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

NX, NY, VIS, U_IN = 512, 128, 0.012, 0.05


def karman_setup():
    th = np.linspace(0, 2 * np.pi, 96, endpoint=False)
    circle = np.stack([np.cos(th), np.sin(th)], 1).astype(np.float32)
    noise = np.random.default_rng(0).uniform(-1e-3, 1e-3, (NX, NY, 2)).astype(np.float32)
    m0 = np.zeros((6, NX, NY), np.float32)
    m0[0] = 1.0
    m0[1] = np.float32(U_IN) + noise[..., 0]
    m0[2] = noise[..., 1]
    return circle, m0


def karman_solver(circle, m0):
    from openhomelbm_b200.lbm import LBM_Solver

    s = LBM_Solver(NX, NY, solid_num=1)
    f = s.flows[0]
    f.vis_shear = VIS
    f.bc_type = [0, 1, 1, 1]
    f.bc_value = np.array([[U_IN, 0.0], [0, 0], [0, 0], [0, 0]], np.float32)
    t = torch.tensor(m0, device=f.device)
    f.moments[0].copy_(t)
    f.moments[1].copy_(t)
    f.configure_solid(0, circle, (128.0, 64.0), angle=0.0, scale=12.0 / 512.0)
    return s


def test_karman_2000_steps_drag_lift_and_moments():
    g = load_golden("karman_cfg1")
    circle, m0 = karman_setup()
    s = karman_solver(circle, m0)
    f = s.flows[0]
    steps = 2000
    loads = torch.zeros((steps, 3), dtype=torch.float32, device=f.device)
    m100 = None
    for k in range(steps):
        s.step()
        loads[k, 0] = f.solid_forcex[0]
        loads[k, 1] = f.solid_forcey[0]
        loads[k, 2] = f.torque[0]
        if k == 99:
            m100 = f.cur.cpu().numpy()
    got = loads.cpu().numpy().astype(np.float64)

    # moments at step 100 against the oracle in binary32 and binary64
    mr = float(f.solid_max_radius[0].item())
    sol = lambda dt: orc.Solids2D(line=circle[None], line_num=np.array([96]), position=np.array([[128.0, 64.0]]),
                                  angle=np.zeros(1), scale=np.array([np.float32(12.0 / 512.0)]),
                                  mass_center=np.zeros((1, 2)), max_radius=np.array([mr])).cast(dt)
    flag = orc.border_flags_2d(NX, NY)
    bc = dict(bc_type=[0, 1, 1, 1], bc_value=[[U_IN, 0.0], [0, 0], [0, 0], [0, 0]], flag=flag, nthreads=0)
    m, p = m0.copy(), m0.copy()
    m64, p64 = m0.astype(np.float64), m0.astype(np.float64)
    s32, s64 = sol(np.float32), sol(np.float64)
    for _ in range(100):
        new, _ = orc.step_2d(m, p, vis_shear=np.float32(VIS), solids=s32, **bc)
        m, p = new, m
        new, _ = orc.step_2d(m64, p64, vis_shear=float(np.float32(VIS)), solids=s64, dtype=np.float64, **bc)
        m64, p64 = new, m64
    own = orc.rel_l2(m, m64)
    print(f"\nKarman step 100: rel L2 of the kernel vs the binary32 oracle {orc.rel_l2(m100, m)}; "
          f"the binary32 oracle's own vs binary64 {own}")
    msgs = orc.check_parity(m100, m, m64, tol=max(1e-5, 3 * max(own.values())))
    assert not msgs, (msgs, own)

    ref32, ref64 = g["loads_f32"].astype(np.float64), g["loads_f64"]
    drag_mean = ref64[:, 0].mean()
    assert abs(got[:, 0].mean() - drag_mean) <= 0.01 * abs(drag_mean), (got[:, 0].mean(), drag_mean)
    assert abs(got[:, 1].mean() - ref64[:, 1].mean()) <= 0.01 * abs(drag_mean)
    for k, name in enumerate(("drag", "lift", "torque")):
        err = np.abs(got[:, k] - ref64[:, k]).max()
        ref_err = np.abs(ref32[:, k] - ref64[:, k]).max()
        assert err <= 3 * ref_err + 1e-7, (name, err, ref_err)
