"""Oracle fixture of the D2Q9 Karman configuration (512 x 128, Re = 100).

The reference's own solver cannot run here (it needs NVIDIA Warp), so the fixture comes from
the oracle (oracle/homelbm_oracle.cpp), which reproduces the reference's kernels bit for bit
on the golden cases. Set-up, as the reference's Karman environment would configure it:

* grid 512 x 128, InitBoundary walls, bc_type (0, 1, 1, 1) with inflow (0.05, 0) on the left
  and zero gradient elsewhere (the closest the reference has to free-slip top/bottom);
* vis_shear 0.012 (tau 0.536, Re = 0.05 * 24 / 0.012 = 100);
* rho = 1, u = (0.05, 0) + U(-1e-3, 1e-3) per component from numpy default_rng(0) as float32 of
  shape (512, 128, 2), S = 0 (set_uniform_flow_kernel's convention);
* the cylinder: generate_unit_circle_points(96) (envs/lbm/solid_func.py:3-15) configured with
  configure_solid(0, pts, (128, 64), angle=0, scale=12/512): a 96-gon of radius 12.

Saved: drag (solid_forcex), lift (solid_forcey) and torque after every one of the first 2000
steps in binary32 and binary64, and the binary64 run continued to 100000 steps, by when the wake
sheds vortices: its lift and drag every 10 steps and the window statistics the GPU run is
compared with (the last 30000 steps, in the saturated shedding cycle). Run time about 17 minutes
on 8 cores.

    python tests/golden/make_cfg1.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as orc  # noqa: E402

NX, NY, VIS, U_IN = 512, 128, 0.012, 0.05
SHORT, LONG, WINDOW = 2000, 100000, (70000, 100000)


def setup():
    th = np.linspace(0, 2 * np.pi, 96, endpoint=False)
    circle = np.stack([np.cos(th), np.sin(th)], 1).astype(np.float32)
    noise = np.random.default_rng(0).uniform(-1e-3, 1e-3, (NX, NY, 2)).astype(np.float32)
    m0 = np.zeros((6, NX, NY), np.float32)
    m0[0] = 1.0
    m0[1] = np.float32(U_IN) + noise[..., 0]
    m0[2] = noise[..., 1]
    max_dist = max(float(np.hypot(p[0], p[1])) for p in circle)
    max_radius = float(np.float32((max_dist + 2.0 ** 0.5) ** 2))
    return circle, m0, max_radius


def solids(circle, max_radius, dt):
    return orc.Solids2D(line=circle[None], line_num=np.array([96]), position=np.array([[128.0, 64.0]]),
                        angle=np.zeros(1), scale=np.array([np.float32(12.0 / 512.0)]), mass_center=np.zeros((1, 2)),
                        max_radius=np.array([max_radius])).cast(dt)


def run(steps, dtype, record_every=1):
    circle, m0, mr = setup()
    sol = solids(circle, mr, dtype)
    flag = orc.border_flags_2d(NX, NY)
    m, p = m0.astype(dtype), m0.astype(dtype)
    vis = np.float32(VIS) if dtype == np.float32 else float(np.float32(VIS))
    out = []
    for k in range(steps):
        new, loads = orc.step_2d(m, p, vis_shear=vis, bc_type=[0, 1, 1, 1],
                                 bc_value=[[U_IN, 0.0], [0, 0], [0, 0], [0, 0]], flag=flag, solids=sol, dtype=dtype,
                                 nthreads=0)
        m, p = new, m
        if (k + 1) % record_every == 0:
            out.append(loads[0].copy())
    return np.array(out)


def shedding_stats(drag, lift):
    """Mean drag, lift standard deviation and Strouhal number f D / U from the mean period of
    the lift's upward zero crossings (about its mean) in a window, series sampled every step."""
    l = lift - lift.mean()
    up = np.where((l[:-1] < 0) & (l[1:] >= 0))[0]
    period = float(np.diff(up).mean()) if len(up) > 1 else float("nan")
    return {"mean_drag": float(drag.mean()), "lift_std": float(lift.std()), "periods": len(up) - 1,
            "period_steps": period, "strouhal": 24.0 / U_IN / period}


def main():
    t0 = time.time()
    s32 = run(SHORT, np.float32)
    long64 = run(LONG, np.float64)
    s64 = long64[:SHORT]
    a, b = WINDOW
    st = shedding_stats(long64[a:b, 0], long64[a:b, 1])
    np.savez_compressed(os.path.join(HERE, "karman_cfg1.npz"), loads_f32=s32.astype(np.float32),
                        loads_f64=s64, long_drag_every10=long64[9::10, 0].astype(np.float32),
                        long_lift_every10=long64[9::10, 1].astype(np.float32), window=np.array(WINDOW),
                        mean_drag=st["mean_drag"], lift_std=st["lift_std"], period_steps=st["period_steps"],
                        strouhal=st["strouhal"], periods=st["periods"])
    print(f"karman_cfg1: {time.time() - t0:.0f} s, window {WINDOW}: {st}")


if __name__ == "__main__":
    main()
