"""Benchmark of the HOME-LBM D3Q27 step on B200: MLUPS and fraction of the HBM roofline.

Workload: the 3D Taylor-Green vortex, periodic 256^3 box, FP32 moment storage, u0 = 0.04,
Re = 1600 (nu = u0 (256/2pi) / 1600). One step = one stream-collide of the whole domain.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

Prints one JSON line (rank 0). Under torchrun each rank steps its own replica of the
domain (the worlds of the reference never interact, so the path shards without a
collective); the timed region is bracketed by a barrier and device synchronisation and the
slowest rank's time is used.

``--impl reference`` times the reference algorithm on the host cores instead: the
reference is Python + NVIDIA Warp, Warp is not installable on this machine, so the CPU arm
runs the C++ restatement of the reference kernels (oracle/, all host threads) on a bounded
slab of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "D3Q27 MLUPS (256^3 periodic Taylor-Green, FP32)"
UNIT = "MLUPS"
BYTES_PER_CELL = {"float32": 80, "float16": 40, "bfloat16": 40, "float64": 160}


# ----------------------------------------------------------------------------- helpers
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (read + write) per cell of one stream-collide launch, from one ncu capture of
# the 256^3 bench workload (profiles/d3q27_stream_collide_tma_256_dram.md).
DRAM_BYTES_PER_CELL = {"float32": 1320.1e6 / 256 ** 3, "float16": 643.2e6 / 256 ** 3}


def profile_traffic(n, storage):
    """dram bytes per launch of the stream-collide kernel (scaled by the cells per launch)."""
    per_cell = DRAM_BYTES_PER_CELL.get(storage)
    return None if per_cell is None else per_cell * n ** 3


class ClockSampler:
    """nvidia-smi clocks and throttle reasons around the timed region, every 100 ms, each
    sample with nvidia-smi's own timestamp (the pipe delivers lines in bursts). The caller keeps
    the GPU loaded before and after the timed steps, so that a timed region shorter than the
    sampling period still has a sample under load on each side."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def samples(self):
        """(unix time, sm MHz, max sm MHz, set of active reasons) per parsed line."""
        import datetime

        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        out = []
        for ln in list(self.lines):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                t = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                sm, mx = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            out.append((t, sm, mx, {n for n, v in zip(names, parts[6:10]) if v.lower().startswith("active")}))
        return out

    def seen_after(self, t: float) -> bool:
        return any(s[0] >= t for s in self.samples())

    def summary(self, t_open: float, t_close: float):
        """The samples inside [t_open, t_close]; if the region was shorter than the sampling
        period, the nearest loaded sample on each side of it."""
        ss = self.samples()
        inside = [s for s in ss if t_open <= s[0] <= t_close]
        window = "timed region"
        if not inside:
            before = [s for s in ss if s[0] < t_open][-1:]
            after = [s for s in ss if s[0] > t_close][:1]
            inside, window = before + after, "nearest sample on each side (timed region shorter than the 100 ms period)"
        if not inside:
            return None
        reasons = set().union(*(s[3] for s in inside))
        return {"sm_mhz": float(np.median([s[1] for s in inside])), "sm_max_mhz": float(max(s[2] for s in inside)),
                "reasons": sorted(reasons), "samples": len(inside), "window": window}


CPU_SLAB_PLANES = 8  # x planes of the periodic slab both CPU legs time


def tgv_slab(n, nx, u0=0.04):
    """The first nx x planes of the n^3 Taylor-Green initial state (float32 moments), as a
    periodic slab: the CPU legs time the same per-cell work on a bounded sample."""
    x = 2 * np.pi * np.arange(n) / n
    Y, Z = np.meshgrid(x, x, indexing="ij")
    X = (2 * np.pi * np.arange(nx) / n)[:, None, None]
    ux = u0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    uy = -u0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    uz = np.zeros_like(ux)
    rho = 1 + 3 * (u0 ** 2 / 16) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2)
    return np.stack([rho, ux, uy, uz, ux * ux, uy * uy, uz * uz, ux * uy, ux * uz, uy * uz]).astype(np.float32)


class CpuSlab:
    """The oracle (C++ restatement of the reference's stream_and_collide_3d) stepping a periodic
    slab of the workload on every host thread. The oracle splits a step over (x, y) rows, so
    each of the threads gets work (2048 rows at 256^2)."""

    def __init__(self, n, nx=CPU_SLAB_PLANES, u0=0.04):
        from oracle import oracle as orc

        self.orc = orc
        self.threads = orc.max_threads()
        self.n, self.nx = n, nx
        self.m = tgv_slab(n, nx, u0)
        self.prev = self.m.copy()
        self.vis = np.float32(u0 * (n / (2 * np.pi)) / 1600.0)
        self.cells = nx * n * n

    @property
    def cores(self):
        return min(self.threads, self.nx * self.n)

    def step(self):
        new, _ = self.orc.step_3d(self.m, self.prev, vis_shear=self.vis, periodic=True, nthreads=self.threads)
        self.m, self.prev = new, self.m

    def sample(self):
        return (f"one stream-collide per step of a periodic {self.nx}x{self.n}x{self.n} slab of the {self.n}^3 "
                f"workload on {self.cores} host threads split over (x, y) rows (C++ restatement of the reference's "
                f"stream_and_collide_3d; Warp is not installable here)")


def cpu_baseline(n_yz, budget_s=12.0):
    """The oracle on a periodic slab of the workload for about budget_s seconds; MLUPS and the
    sample description."""
    slab = CpuSlab(n_yz)
    slab.step()  # warm-up
    steps = 0
    t0 = time.perf_counter()
    while True:
        slab.step()
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": slab.cells * steps / dt / 1e6, "unit": UNIT, "cores": slab.cores, "kind": "port",
            "sample": f"{steps} steps ({dt:.1f} s): " + slab.sample()}


# ----------------------------------------------------------------------------- arms
# ----------------------------------------------------------------------------- replicas
def init_replicas(backend: str = "nccl", timeout_s: float = 300.0):
    """(rank, world, torch.distributed or None) from the launcher's RANK / WORLD_SIZE /
    MASTER_* environment; one process per GPU, each stepping its own replica."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world <= 1:
        return rank, world, None
    import datetime

    import torch.distributed as tdist

    tdist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, tdist


def max_over_ranks(x: float, dist, device=None) -> float:
    """The largest x over the ranks (the slowest replica's time); x itself without a group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, cells_per_replica: int, steps: int, seconds: float) -> float:
    """Whole-job MLUPS: every replica's cell updates over the slowest replica's time."""
    return world * cells_per_replica * steps / seconds / 1e6


def run_reference(args, rank, world):
    if rank != 0:
        return None
    n = args.n
    slab = CpuSlab(n)
    for _ in range(args.warmup):
        slab.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        slab.step()
    dt = time.perf_counter() - t0
    value = slab.cells * args.steps / dt / 1e6
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (Taylor-Green initial state)",
            "config": {"workload": f"D3Q27 Taylor-Green vortex {n}^3 periodic, FP32", "u0": 0.04,
                       "Re": 1600, "sample_cells": slab.cells},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": slab.cores, "kind": "port",
                             "sample": slab.sample()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_ours(args, rank, world, dist):
    import torch

    from openhomelbm_b200 import _lib
    from openhomelbm_b200.lbm3d import LBM_Solver3D

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    _lib.set_tuning("d3q27_kernel", args.kernel)
    _lib.set_tuning("d3q27_chunks", args.chunks)
    _lib.set_tuning("d3q27_stages", args.stages)
    n = args.n
    storage = args.storage
    u0 = 0.04
    vis = u0 * (n / (2 * np.pi)) / 1600.0
    s = LBM_Solver3D(n, n, n, solid_num=1, periodic=True, storage=storage, device=dev,
                     u_scale=u0, s_scale=u0 * u0)
    s.set_viscosity(vis)
    s.init_tgv(u0)
    f = s.flows[0]
    cells = n ** 3
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------------------------------------------------------- device-resident timing
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        # warm-up: at least W steps, continued (at most 5 s) until the clock sampler has
        # logged the GPU under this load
        t_warm = time.time()
        done = 0
        while done < max(args.warmup, 3) or (clk.proc is not None and time.time() - t_warm < 5.0 and
                                             (done % 32 or not clk.seen_after(t_warm + 0.15))):
            s.step()
            done += 1
            if done % 64 == 0:
                torch.cuda.synchronize()
        barrier()
        t_open = time.time()
        start.record(stream)
        for _ in range(args.steps):
            s.step()
        end.record(stream)
        barrier()
        t_close = time.time()
        # keep the load (untimed) for one sampling period, so a sample follows the region
        while time.time() - t_close < 0.15:
            s.step()
            torch.cuda.synchronize()
        time.sleep(0.15)
    ms = max_over_ranks(start.elapsed_time(end), dist, dev)
    ms_step = ms / args.steps
    value = job_rate(world, cells, args.steps, ms / 1e3)

    # ---------------------------------------------------------------- end to end, host buffers
    # Through the public API (LBM_Solver3D.step -> libhomelbm): the job's input field is
    # uploaded from pinned host memory inside the timed region, every step's result (the
    # binary64 mass and the health word) is copied to pinned host memory and waited for by
    # the host before the next step, and the final field is downloaded at the end.
    ke = args.steps if args.e2e_steps <= 0 else min(args.steps, args.e2e_steps)  # default: the same K steps
    init_host = f.cur.detach().to("cpu").pin_memory()
    out_host = torch.empty_like(init_host).pin_memory()
    mass_host = torch.empty(ke, dtype=torch.float64).pin_memory()
    health_host = torch.empty(ke, dtype=torch.int32).pin_memory()
    s.diagnostics = True
    s.step()
    barrier()
    parity0 = f.parity
    t0 = time.perf_counter()
    f.cur.copy_(init_host, non_blocking=True)
    for k in range(ke):
        s.step()
        mass_host[k:k + 1].copy_(s.mass[0:1], non_blocking=True)
        health_host[k:k + 1].copy_(s.health[0:1], non_blocking=True)
        stream.synchronize()
    out_host.copy_(f.cur, non_blocking=True)
    stream.synchronize()
    e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e = job_rate(world, cells, ke, e_s)
    field_bytes = init_host.numel() * init_host.element_size()
    health = int(health_host.max().item())
    s.diagnostics = False
    # the end-to-end result against the same steps run resident on the device (diagnostics off)
    f.parity = parity0
    f.cur.copy_(init_host)
    for _ in range(ke):
        s.step()
    e2e_same = bool(torch.equal(f.cur, out_host.to(dev)))

    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    bpc = BYTES_PER_CELL[storage]
    achieved = bpc * cells / (ms_step / 1e3) / 1e9
    traffic = profile_traffic(n, storage)
    out = {
        "metric": METRIC if storage == "float32" else METRIC.replace("FP32", storage),
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (Taylor-Green initial state)",
        "config": {"workload": f"D3Q27 Taylor-Green vortex {n}^3 periodic, {storage} storage, one stream-collide "
                               f"per step", "u0": u0, "Re": 1600, "vis_shear": vis,
                   "kernel": {0: "auto", 1: "async-copy", 2: "tma"}[args.kernel], "chunks": args.chunks, "stages": args.stages,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 "
                   f"({cells * bpc / 1e9:.2f} GB moved per step vs 126 MB L2)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_cell": bpc},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": field_bytes / ke,
                "d2h_bytes_per_step": field_bytes / ke + 12, "steps": ke,
                "field_equals_device_run": e2e_same,
                "note": f"{ke} steps through LBM_Solver3D.step: input field uploaded from pinned host memory, "
                        "each step's mass and health words copied to pinned host memory and awaited by the "
                        "host, final field downloaded; host wall clock"},
        "gpu_launches": args.steps * (1 + (0 if f.periodic else 3)),
        "warmup_steps_run": done,
        "health_nonfinite_cells": health,
    }
    c = clk.summary(t_open, t_close)
    if c is not None:
        out["clocks"] = c
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(n, budget_s=args.cpu_budget)
    return out


# ----------------------------------------------------------------------------- precision form
def tgv_diagnostics(f, n):
    """Kinetic energy 1/2 <rho |u|^2> and enstrophy 1/2 <|curl u|^2> (periodic central
    differences, unit lattice spacing) of a world, in binary64."""
    import torch

    m = f.decoded().double()
    rho, u = m[0], m[1:4]
    ke = 0.5 * float((rho * (u * u).sum(0)).mean())

    def d(a, axis):
        return 0.5 * (torch.roll(a, -1, axis) - torch.roll(a, 1, axis))

    wx = d(u[2], 1) - d(u[1], 2)
    wy = d(u[0], 2) - d(u[2], 0)
    wz = d(u[1], 0) - d(u[0], 1)
    ens = 0.5 * float((wx * wx + wy * wy + wz * wz).mean())
    return ke, ens


def run_precision(args, n=None, steps=None, every=10):
    """The precision form: the Taylor-Green vortex with float64 (the accuracy oracle, same
    kernels in binary64), float32, float16 and bfloat16 storage. Each run records kinetic
    energy and enstrophy every ``every`` steps and the binary64 mass sum every step; the reduced
    forms report their velocity L2 error against the float64 run and their MLUPS against
    the float32 run (timed separately, diagnostics off)."""
    import torch

    from openhomelbm_b200.lbm3d import LBM_Solver3D

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n = args.n if n is None else n
    steps = args.steps if steps is None else steps
    u0 = 0.04
    vis = u0 * (n / (2 * np.pi)) / 1600.0
    cells = n ** 3
    res, u_ref = {}, None
    for storage in ("float64", "float32", "float16", "bfloat16"):
        s = LBM_Solver3D(n, n, n, solid_num=1, periodic=True, storage=storage, device=dev, u_scale=u0,
                         s_scale=u0 * u0)
        s.set_viscosity(vis)
        s.init_tgv(u0)
        f = s.flows[0]
        s.diagnostics = True
        ke, ens, mass = [], [], torch.zeros(steps, dtype=torch.float64, device=dev)
        k0, e0 = tgv_diagnostics(f, n)
        ke.append(k0)
        ens.append(e0)
        for k in range(steps):
            s.step()
            mass[k] = s.mass[0]
            if (k + 1) % every == 0:
                kk, ee = tgv_diagnostics(f, n)
                ke.append(kk)
                ens.append(ee)
        s.diagnostics = False
        u = f.decoded()[1:4].double()
        rec = {f"ke_every_{every}": [round(x, 12) for x in ke],
               f"enstrophy_every_{every}": [round(x, 12) for x in ens],
               "mass_first": float(mass[0]), "mass_last": float(mass[-1]),
               "mass_rel_drift": float((mass[-1] - mass[0]) / mass[0]), "health": int(s.health[0])}
        if u_ref is None:
            u_ref = u.clone()
        else:
            rec["u_l2_vs_float64"] = float(torch.linalg.vector_norm(u - u_ref) / torch.linalg.vector_norm(u_ref))
        del u
        # throughput, diagnostics off
        for _ in range(3):
            s.step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        timed = min(steps, 200)
        a.record()
        for _ in range(timed):
            s.step()
        b.record()
        torch.cuda.synchronize()
        rec["mlups"] = cells * timed / (a.elapsed_time(b) / 1e3) / 1e6
        res[storage] = rec
        del s, f
        torch.cuda.empty_cache()
    f32 = res["float32"]["mlups"]
    for st in ("float16", "bfloat16"):
        res[st]["mlups_vs_float32"] = res[st]["mlups"] / f32
    return {"metric": f"D3Q27 velocity L2 vs float64 (Taylor-Green {n}^3, {steps} steps, reduced storage)",
            "value": res["float16"]["u_l2_vs_float64"], "unit": "relative L2", "higher_is_better": False,
            "n_gpus": 1, "steps": steps, "workload": "precision", "dtype": "f32 arithmetic",
            "data": "synthetic (Taylor-Green initial state)",
            "config": {"workload": f"D3Q27 Taylor-Green vortex {n}^3 periodic; float64 / float32 / float16 / bfloat16 "
                                   "storage (rho - 1, u / u0, (S - u u) / u0^2)", "u0": u0, "Re": 1600,
                       "vis_shear": vis, "diagnostics_every": every},
            "results": res}


# ----------------------------------------------------------------------------- Karman form
def shedding_stats(drag, lift, diameter=24.0, u_in=0.05):
    """Mean drag, lift standard deviation and Strouhal number f D / U from the mean period of
    the lift's upward zero crossings about its mean (series sampled every step)."""
    l = lift - lift.mean()
    up = np.where((l[:-1] < 0) & (l[1:] >= 0))[0]
    period = float(np.diff(up).mean()) if len(up) > 1 else float("nan")
    return {"mean_drag": float(drag.mean()), "lift_std": float(lift.std()), "periods": int(len(up) - 1),
            "period_steps": period, "strouhal": diameter / u_in / period}


def run_karman(args, cpu=True):
    """The D2Q9 Karman configuration: 512 x 128, 96-gon cylinder of radius 12 at (128, 64),
    inflow (0.05, 0), zero gradient elsewhere, nu = 0.012 (Re 100), rho = 1 and u = inflow plus
    seeded +-1e-3 noise. 100000 steps on the GPU with drag and lift recorded every step; the
    shedding statistics over steps 70000-100000 against the binary64 oracle run of the same
    configuration (tests/golden/karman_cfg1.npz, made by tests/golden/make_cfg1.py)."""
    import torch

    from openhomelbm_b200.lbm import LBM_Solver

    torch.cuda.set_device(0)
    nx, ny, vis, u_in = 512, 128, 0.012, 0.05
    th = np.linspace(0, 2 * np.pi, 96, endpoint=False)
    circle = np.stack([np.cos(th), np.sin(th)], 1).astype(np.float32)
    noise = np.random.default_rng(0).uniform(-1e-3, 1e-3, (nx, ny, 2)).astype(np.float32)
    m0 = np.zeros((6, nx, ny), np.float32)
    m0[0] = 1.0
    m0[1] = np.float32(u_in) + noise[..., 0]
    m0[2] = noise[..., 1]
    s = LBM_Solver(nx, ny, solid_num=1)
    f = s.flows[0]
    f.vis_shear = vis
    f.bc_type = [0, 1, 1, 1]
    f.bc_value = np.array([[u_in, 0.0], [0, 0], [0, 0], [0, 0]], np.float32)
    t = torch.tensor(m0, device=f.device)
    f.moments[0].copy_(t)
    f.moments[1].copy_(t)
    f.configure_solid(0, circle, (128.0, 64.0), angle=0.0, scale=12.0 / 512.0)
    steps = args.karman_steps
    loads = torch.zeros((steps, 2), dtype=torch.float32, device=f.device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for k in range(steps):
        s.step()
        loads[k, 0] = f.solid_forcex[0]
        loads[k, 1] = f.solid_forcey[0]
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    got = loads.cpu().numpy().astype(np.float64)
    g = np.load(os.path.join(ROOT, "tests", "golden", "karman_cfg1.npz"))
    w0, w1 = (int(v) for v in g["window"])
    ours = shedding_stats(got[w0:w1, 0], got[w0:w1, 1]) if steps >= w1 else None
    ref = {k: float(g[k]) for k in ("mean_drag", "lift_std", "strouhal", "period_steps")}
    rel = ({k: ours[k] / ref[k] - 1.0 for k in ("mean_drag", "lift_std", "strouhal")} if ours else None)
    out = {"metric": "D2Q9 Karman wake (512x128, Re 100) Strouhal number vs binary64 oracle",
           "value": ours["strouhal"] if ours else None, "unit": "St", "higher_is_better": None, "n_gpus": 1,
           "workload": "karman", "steps": steps, "dtype": "f32", "data": "synthetic (seeded inflow noise)",
           "window": [w0, w1], "ours": ours, "oracle_f64": ref, "relative_difference": rel,
           "mlups": nx * ny * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps,
           "config": {"workload": "D2Q9 512x128, 96-gon cylinder r=12 at (128,64), inflow 0.05, nu 0.012, bc 0,1,1,1",
                      "recorded": "drag (solid_forcex) and lift (solid_forcey) every step, device-side"}}
    if not cpu:
        return out
    # CPU baseline: the oracle (C++ restatement of the reference kernels, all host threads)
    from oracle import oracle as orc

    mr = float(f.solid_max_radius[0].item())
    sol = orc.Solids2D(line=circle[None], line_num=np.array([96]), position=np.array([[128.0, 64.0]]), angle=np.zeros(1),
                       scale=np.array([np.float32(12.0 / 512.0)]), mass_center=np.zeros((1, 2)),
                       max_radius=np.array([mr])).cast(np.float32)
    flag = orc.border_flags_2d(nx, ny)
    mm, pp = m0.copy(), m0.copy()
    threads = orc.max_threads()
    n_cpu, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < args.cpu_budget:
        new, _ = orc.step_2d(mm, pp, vis_shear=np.float32(vis), bc_type=[0, 1, 1, 1],
                             bc_value=[[u_in, 0.0], [0, 0], [0, 0], [0, 0]], flag=flag, solids=sol, nthreads=threads)
        mm, pp = new, mm
        n_cpu += 1
    cpu_s = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": nx * ny * n_cpu / cpu_s / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
                           "sample": f"{n_cpu} steps of the same 512x128 domain with its cylinder ({cpu_s:.1f} s, "
                                     "C++ restatement of the reference's D2Q9 kernels, not Warp)"}
    return out


# ----------------------------------------------------------------------------- serving form
def run_serve(args, batched_variant=True):
    """The serving form: Poisson arrivals of mesh-coupled D3Q27 domains (sides log-uniform in
    64-192, rounded to multiples of 32; a 5-segment swimmer of 1800 triangles; 8 LBM substeps
    per control step, 100 control steps per request). The served engine (float16 storage,
    resident fields, one CUDA graph per domain control step, concurrent domains) against the
    plain solver one request at a time (float32), on the same request set."""
    import torch

    from openhomelbm_b200 import serving

    torch.cuda.set_device(0)
    reqs = serving.poisson_requests(args.requests, args.rate, seed=7, control_steps=args.control_steps)
    warm = [serving.Request(10 ** 6, 64, 1, 0.0, control_steps=2, substeps=8)]
    serving.run_plain(warm)
    serving.ServeEngine(storage="float16", max_active=1).run(warm, realtime=False)
    torch.cuda.synchronize()
    plain = serving.run_plain(reqs, storage="float32")
    engine = serving.ServeEngine(storage="float16", max_active=args.slots, budget_bytes=150e9)
    served = engine.run(reqs)
    # the same requests with one stream-collide launch per substep over all active domains
    batched = (serving.ServeEngine(storage="float16", max_active=args.slots, budget_bytes=150e9,
                                   batched=True).run(reqs) if batched_variant else None)
    # agreement of the served float16 loads with the plain float32 loads, request by request
    errs = []
    for r in reqs:
        a, b = served.results[r.rid].astype(np.float64), plain.results[r.rid].astype(np.float64)
        errs.append(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)))
    cells = sum(r.side ** 3 * r.control_steps * r.substeps for r in reqs)
    sides = [r.side for r in reqs]
    # accuracy of the served float16 form: final velocity fields against float64 storage (the
    # same kernels in binary64) for two swimmers of each size up to 160
    acc_reqs = [serving.Request(100 + k, side, 1000 + k, 0.0, control_steps=args.control_steps)
                for k, side in enumerate((64, 96, 128, 160) * 2)]
    f64 = serving.ServeEngine(storage="float64", max_active=8, keep_fields=True).run(acc_reqs, realtime=False)
    f16 = serving.ServeEngine(storage="float16", max_active=8, keep_fields=True).run(acc_reqs, realtime=False)
    u_l2 = {}
    for r in acc_reqs:
        e = float(np.linalg.norm(f16.fields[r.rid] - f64.fields[r.rid]) / np.linalg.norm(f64.fields[r.rid]))
        u_l2.setdefault(str(r.side), []).append(e)
    all_e = [e for v in u_l2.values() for e in v]
    return {"metric": "served env-steps/s (D3Q27 mesh-coupled domains, float16 storage, continuous batching)",
            "value": served.env_steps_per_s, "unit": "env-steps/s", "higher_is_better": True, "n_gpus": 1,
            "workload": "serve", "dtype": "f32 arithmetic, f16 storage", "data": "synthetic (seeded Poisson requests)",
            "vs_plain": served.env_steps_per_s / plain.env_steps_per_s,
            "served": {"env_steps_per_s": served.env_steps_per_s, "p50_ms": served.pct(50) * 1e3,
                       "p99_ms": served.pct(99) * 1e3, "p99_over_p50": served.pct(99) / served.pct(50),
                       "wall_s": served.wall_s, "max_active": served.max_active,
                       "mlups": cells / served.wall_s / 1e6},
            "served_batched_stream_collide": ({"env_steps_per_s": batched.env_steps_per_s,
                                               "p50_ms": batched.pct(50) * 1e3, "p99_ms": batched.pct(99) * 1e3}
                                              if batched is not None else None),
            "plain": {"env_steps_per_s": plain.env_steps_per_s, "p50_ms": plain.pct(50) * 1e3,
                      "p99_ms": plain.pct(99) * 1e3, "wall_s": plain.wall_s, "mlups": cells / plain.wall_s / 1e6},
            "loads_rel_l2_f16_vs_plain_f32": {"median": float(np.median(errs)), "max": float(np.max(errs))},
            "u_l2_f16_vs_f64_by_side": u_l2,
            "u_l2_f16_vs_f64": {"median": float(np.median(all_e)), "max": float(np.max(all_e))},
            "config": {"requests": len(reqs), "rate_per_s": args.rate, "control_steps": args.control_steps,
                       "substeps": 8, "slots": args.slots, "hbm_budget_gb": 150, "served_x_chunks": engine.x_chunks,
                       "served_link_blocks": engine.link_blocks,
                       "sides": {str(k): sides.count(k) for k in sorted(set(sides))},
                       "triangles_per_body": 1800, "segments": serving.SEGMENTS}}


def run_batch(args):
    """The batching form: args.worlds D2Q9 worlds (nx ~ logU[256, 1024], ny ~ logU[128, 512] from
    default_rng(args.seed)), each with an 8-capsule swimmer (body 64 cells, capsule radius 4) on
    a prescribed travelling wave, float16 storage, 8 substeps per control step. A substep is one
    launch per phase for all worlds, the stream phase one persistent launch over the tile
    work-list (tile shape and grid from the autotuner); a control step is one CUDA graph. The
    same worlds one at a time through the plain float32 solver are the baseline. The tile
    kernel is also timed alone (stream phase of all worlds, CUDA events; the batch's fields,
    ~10 M cells x 24 B, exceed L2) for its HBM roofline: 24 B per cell update (6 float16
    moments read and written)."""
    import torch

    from openhomelbm_b200 import _lib, batching

    torch.cuda.set_device(0)
    specs = batching.swimmer_specs(args.worlds, seed=args.seed)
    tuner = batching.TileAutotuner()
    sb = batching.SwimmerBatch2D(specs, storage="float16", autotuner=tuner)
    sb.run(2)  # warm-up
    K = args.batch_control_steps
    stats = sb.run(K)
    b, st = sb.batch, _lib.stream_ptr()
    reps = 50
    for _ in range(5):
        b.launch(0, st, phases=_lib.HL_PHASE_STREAM, any_solid=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        b.launch(0, st, phases=_lib.HL_PHASE_STREAM, any_solid=False)
    e1.record()
    torch.cuda.synchronize()
    t_kernel = e0.elapsed_time(e1) / reps * 1e-3
    cells = b.cells()
    achieved = cells * 24 / t_kernel / 1e9
    peak, peak_kind = measured_peaks()
    # the plain run covers the batch's warm-up control steps too; compare the same steps
    plain = batching.run_sequential_plain(specs, K + 2)
    a, p = stats.loads.astype(np.float64), plain.loads[2:].astype(np.float64)
    rel = float(np.linalg.norm(a - p) / np.linalg.norm(p))
    cfg = stats.config
    table = {f"{c.tile_x}x{c.tile_y}/{c.ctas}": round(ms * 1e3, 1) for c, ms in sorted(stats.tune_table.items(),
                                                                                       key=lambda kv: kv[1])}
    return {"metric": "batched MLUPS (uneven D2Q9 worlds with capsule swimmers, float16 storage)",
            "value": stats.mlups, "unit": "MLUPS", "higher_is_better": True, "n_gpus": 1, "workload": "batch",
            "dtype": "f32 arithmetic, f16 storage", "data": "synthetic (seeded sizes and swimmers)",
            "vs_sequential": stats.mlups / plain.mlups,
            "batched": {"mlups": stats.mlups, "ms_per_control_step": stats.wall_s / K * 1e3,
                        "p50_ms": float(np.percentile(stats.latencies_s, 50)) * 1e3,
                        "p99_ms": float(np.percentile(stats.latencies_s, 99)) * 1e3,
                        "tile": [cfg.tile_x, cfg.tile_y], "ctas": cfg.ctas},
            "sequential_plain": {"mlups": plain.mlups,
                                 "ms_per_control_step_all_worlds": plain.wall_s / (K + 2) * 1e3},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "kernel": "stream_tiles_kernel",
                         "us_per_launch": t_kernel * 1e6, "bytes_per_cell": 24},
            "autotuner_us_per_launch": table,
            "loads_rel_l2_f16_batch_vs_plain_f32": rel,
            "config": {"workload": "batch", "worlds": len(specs), "seed": args.seed, "cells": cells,
                       "control_steps": K, "substeps": 8, "capsules": 8, "storage": "float16",
                       "l2": "inputs larger than L2"}}


def karman_leg(args):
    """configs[0] for the default line: the Karman wake's Strouhal number, mean drag and lift
    spread over steps 70000-100000 against the binary64 oracle run of the same configuration."""
    r = run_karman(args, cpu=False)
    return {k: r[k] for k in ("metric", "value", "unit", "steps", "window", "ours", "oracle_f64",
                              "relative_difference", "mlups", "config")}


def precision_leg(args):
    """configs[2] for the default line: the Taylor-Green vortex at 512^3 for 2000 steps in float64,
    float32, float16 and bfloat16 storage; velocity L2 against float64, mass drift, MLUPS, and the
    kinetic energy every 100 steps."""
    r = run_precision(args, n=512, steps=2000, every=100)
    res = {}
    for st, v in r["results"].items():
        res[st] = {k: v[k] for k in ("mlups", "mass_rel_drift", "health") if k in v}
        for k in ("u_l2_vs_float64", "mlups_vs_float32"):
            if k in v:
                res[st][k] = v[k]
        res[st]["ke_every_100"] = v["ke_every_100"]
    return {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "results": res,
            "config": dict(r["config"], diagnostics_every=100)}


def serve_leg(args):
    """The serving form's figures for the default line: served (float16, continuous batching)
    against the plain float32 solver one request at a time, on the same seeded requests."""
    r = run_serve(args, batched_variant=False)
    keep = ("env_steps_per_s", "p50_ms", "p99_ms", "p99_over_p50", "wall_s", "max_active")
    return {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "vs_plain": r["vs_plain"],
            "served": {k: r["served"][k] for k in keep},
            "plain": {k: r["plain"][k] for k in ("env_steps_per_s", "p50_ms", "p99_ms", "wall_s")},
            "u_l2_f16_vs_f64": r["u_l2_f16_vs_f64"], "loads_rel_l2_f16_vs_plain_f32": r["loads_rel_l2_f16_vs_plain_f32"],
            "config": r["config"]}


def batch_leg(args):
    """The batching form's figures for the default line: 64 uneven D2Q9 worlds in one persistent
    launch per substep, against the same worlds solved one at a time."""
    r = run_batch(args)
    return {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "vs_sequential": r["vs_sequential"],
            "batched": r["batched"], "sequential_plain": r["sequential_plain"], "roofline": r["roofline"],
            "loads_rel_l2_f16_batch_vs_plain_f32": r["loads_rel_l2_f16_batch_vs_plain_f32"], "config": r["config"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps of the end-to-end run (0: --steps)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--storage", default="float32", choices=list(BYTES_PER_CELL))
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel", type=int, default=0, help="0 auto, 1 async-copy kernel, 2 TMA kernel")
    ap.add_argument("--chunks", type=int, default=0, help="x split per tile column (0 automatic)")
    ap.add_argument("--stages", type=int, default=0, help="TMA pipeline stages (0 automatic)")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "precision", "serve", "karman", "batch"],
                    help="tgv: the headline throughput line; precision: float64/32/16/bf16 accuracy form; "
                         "serve: served vs plain mesh-coupled domains; karman: D2Q9 wake vs the oracle; "
                         "batch: uneven D2Q9 worlds in one persistent launch vs sequential plain solves")
    ap.add_argument("--worlds", type=int, default=64, help="batch: number of worlds")
    ap.add_argument("--seed", type=int, default=0, help="batch: seed of the world sizes and swimmers")
    ap.add_argument("--batch-control-steps", type=int, default=20, help="batch: timed control steps")
    ap.add_argument("--requests", type=int, default=48, help="serve: number of requests")
    ap.add_argument("--karman-steps", type=int, default=100000, help="karman: GPU steps")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: Poisson arrival rate (requests/s)")
    ap.add_argument("--control-steps", type=int, default=100, help="serve: control steps per request")
    ap.add_argument("--slots", type=int, default=32, help="serve: concurrently resident domains")
    ap.add_argument("--no-legs", action="store_true",
                    help="tgv: leave out the serve and batch legs of the default line")
    args = ap.parse_args()
    legs = args.workload == "tgv" and args.impl == "ours" and not args.no_legs and \
        int(os.environ.get("WORLD_SIZE", "1")) == 1
    if args.workload == "serve" or legs:
        # a hardware work queue per resident domain's stream (before any CUDA call)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl == "reference" and rank != 0:
        return  # the CPU arm runs on rank 0 only
    if world > 1 and args.impl != "reference":
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        rank, world, dist = init_replicas("nccl")
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world)
        elif args.workload == "precision":
            out = run_precision(args) if rank == 0 else None
        elif args.workload == "serve":
            out = run_serve(args) if rank == 0 else None
        elif args.workload == "karman":
            out = run_karman(args) if rank == 0 else None
        elif args.workload == "batch":
            out = run_batch(args) if rank == 0 else None
        else:
            out = run_ours(args, rank, world, dist)
            if legs and out is not None:
                # the second half of the headline metric (served env-steps/s and latency against
                # the plain solver) and the batching form, measured in the same run
                t0 = time.perf_counter()
                out["serve"] = serve_leg(args)
                out["serve"]["leg_wall_s"] = time.perf_counter() - t0
                t0 = time.perf_counter()
                out["batch"] = batch_leg(args)
                out["batch"]["leg_wall_s"] = time.perf_counter() - t0
                t0 = time.perf_counter()
                out["karman"] = karman_leg(args)
                out["karman"]["leg_wall_s"] = time.perf_counter() - t0
                t0 = time.perf_counter()
                out["precision"] = precision_leg(args)
                out["precision"]["leg_wall_s"] = time.perf_counter() - t0
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
