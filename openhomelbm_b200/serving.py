"""Serving form: a request loop of mesh-coupled D3Q27 domains kept resident on the GPU.

Each request is one RL environment's flow: a cubic domain with a 5-segment swimmer whose yaw
joints follow seeded sinusoids; the caller wants per-segment force and torque after every
control step (``substeps`` LBM steps), for ``control_steps`` control steps.

``ServeEngine`` runs requests with continuous batching: a request that has arrived is admitted
as soon as a slot is free and its fields fit the HBM budget; its fields stay on the device for
its whole life; every active request advances one control step per tick. By default a
domain's whole control step (pose updates, stream-collide, cut links, boundaries and load
copies for all substeps) is captured once into a CUDA graph at admission and each tick
launches every active domain's graph on its own CUDA stream, so the domains' kernels overlap
on the device. With ``batched=True`` each substep is instead ONE stream-collide launch over
every active domain (hl_d3q27_stream_collide_batch: the tiles of all domains share the SMs)
and ONE cut-link pass over all of them (hl_d3q27_solid_links_batch), then the boundaries of
all of them as one launch per wave (hl_d3q27_apply_bc_batch), then each domain's next pose on
its own stream; once the set of active domains has held for two ticks, the whole control step
of the set is one CUDA graph (``TickGraph``). Both give the same results; in the batched form
the cut links and boundaries run between two batched stream-collides instead of behind other
domains' stream-collides. The poses of every domain's next control step are computed on the host
while the tick runs on the device. Admission (allocation, initial state, graph capture)
happens between ticks and counts in the wall time, not in a control step's latency.
``run_plain`` is the baseline: the same requests one at a time through the plain drop-in
solver (LBM_Solver3D, float32 storage), one graph launch per LBM step.

Every domain's result is independent of the others in the mix: the kernels of one domain
read and write only that domain's buffers.
"""
from __future__ import annotations

import contextlib
import ctypes
import gc
import math
import os
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .lbm3d import LBM_Solver3D

SEGMENTS = 5
# One hardware work queue per domain stream: with CUDA's default of 8, the streams of more
# than 8 domains share queues and their graphs run one after another. Effective only when
# this module is imported before the process creates its CUDA context.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


@contextlib.contextmanager
def _capturing():
    """No cyclic garbage collection while a CUDA graph is captured: a collected object that
    owns a CUDA graph would destroy it mid-capture, which invalidates the capture."""
    enabled = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if enabled:
            gc.enable()


@contextlib.contextmanager
def _graph_capture(graph: torch.cuda.CUDAGraph, stream: torch.cuda.Stream):
    """Capture the work issued on ``stream`` into ``graph``, with cyclic GC off (_capturing).

    torch.cuda.graph() would first synchronize the device, run gc.collect() and empty the
    caching allocator. Here that is wrong three times over: the synchronize waits for every
    resident domain's tick in flight, and emptying the cache returns the freed domains' blocks
    to the driver, so the next admissions allocate afresh. Measured on a B200 with 32 resident
    domains: most captures take ~2 ms, but two or three per run took 0.8-0.9 s, which added
    up to 2 s to a 3.6 s run. Capturing directly skips all three; nothing issued here needs
    them."""
    with _capturing(), torch.cuda.stream(stream):
        graph.capture_begin()
        try:
            yield
        finally:
            graph.capture_end()


# ----------------------------------------------------------------------------- bodies
def ellipsoid_mesh(a: float, b: float, c: float, n_lon: int = 20, n_lat: int = 11) -> Tuple[np.ndarray, np.ndarray]:
    """Closed triangle mesh of an ellipsoid with semi-axes (a, b, c) centred at (a, 0, 0), so
    that its joint (the body-frame origin) sits on its back end: 2 n_lon (n_lat - 2) triangles
    (360 for the defaults)."""
    verts = [(0.0, 0.0, 0.0)]  # back pole (x = 0)
    for i in range(1, n_lat - 1):
        th = math.pi * i / (n_lat - 1)
        for j in range(n_lon):
            ph = 2 * math.pi * j / n_lon
            verts.append((a - a * math.cos(th), b * math.sin(th) * math.cos(ph), c * math.sin(th) * math.sin(ph)))
    verts.append((2 * a, 0.0, 0.0))  # front pole
    faces = []
    ring = lambda i, j: 1 + (i - 1) * n_lon + (j % n_lon)
    for j in range(n_lon):
        faces.append((0, ring(1, j + 1), ring(1, j)))
    for i in range(1, n_lat - 2):
        for j in range(n_lon):
            faces.append((ring(i, j), ring(i, j + 1), ring(i + 1, j)))
            faces.append((ring(i, j + 1), ring(i + 1, j + 1), ring(i + 1, j)))
    last = len(verts) - 1
    for j in range(n_lon):
        faces.append((last, ring(n_lat - 2, j), ring(n_lat - 2, j + 1)))
    return np.array(verts, np.float64), np.array(faces, np.int64)


@dataclass
class Swimmer:
    """A chain of SEGMENTS ellipsoids joined by yaw joints. Segment k's body frame has its
    joint at the origin; joint angle k follows amp[k] sin(2 pi freq t + phase[k]) (t in LBM
    steps), and the head's joint is fixed at ``head``. The amplitudes grow towards the tail and
    the frequency is set from a seeded peak wall speed of 0.02-0.04 lattice units per step
    (the bound omega L sum_k amp[k] (SEGMENTS - k) of the tail's speed), well inside the
    low-Mach range of the lattice whatever the domain size."""

    side: int
    seg_len: float
    head: np.ndarray
    amp: np.ndarray
    freq: float
    phase: np.ndarray
    meshes: List[Tuple[np.ndarray, np.ndarray]] = field(default_factory=list)

    @staticmethod
    def make(side: int, rng: np.random.Generator) -> "Swimmer":
        L = 0.1 * side
        meshes = [ellipsoid_mesh(L / 2, 0.18 * L, 0.14 * L) for _ in range(SEGMENTS)]
        head = np.array([0.3 * side, 0.5 * side + rng.uniform(-1, 1), 0.5 * side + rng.uniform(-1, 1)])
        amp = 0.15 * rng.uniform(0.8, 1.2) * (0.2 + 0.2 * np.arange(SEGMENTS))
        v_peak = rng.uniform(0.02, 0.04)
        freq = v_peak / (2 * np.pi * L * float(np.sum(amp * (SEGMENTS - np.arange(SEGMENTS)))))
        return Swimmer(side, L, head, amp, float(freq), rng.uniform(0, 2 * np.pi, SEGMENTS), meshes)

    def poses(self, t: float) -> Tuple[np.ndarray, np.ndarray]:
        """Joint positions (SEGMENTS, 3) and orientations (SEGMENTS, 4) as (w, x, y, z)."""
        pos, quat = self.poses_at(np.array([t], np.float64))
        return pos[0], quat[0]

    def poses_at(self, ts: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        """Poses at every time of ``ts``: positions (T, SEGMENTS, 3), quaternions (T, SEGMENTS, 4).
        Segment k's yaw is the sum of joint angles 0..k; joint k + 1 sits one segment length
        along segment k's axis."""
        ts = np.asarray(ts, np.float64)
        ang = self.amp[None, :] * np.sin(2 * np.pi * self.freq * ts[:, None] + self.phase[None, :])
        yaw = np.cumsum(ang, axis=1)
        step = self.seg_len * np.stack([np.cos(yaw), np.sin(yaw), np.zeros_like(yaw)], axis=2)
        pos = self.head[None, None, :] + np.concatenate([np.zeros_like(step[:, :1]), np.cumsum(step, axis=1)[:, :-1]],
                                                          axis=1)
        quat = np.stack([np.cos(yaw / 2), np.zeros_like(yaw), np.zeros_like(yaw), np.sin(yaw / 2)], axis=2)
        return pos.astype(np.float32), quat.astype(np.float32)


@dataclass
class Request:
    """One environment: domain side, body seed, arrival time (s after the loop starts)."""

    rid: int
    side: int
    seed: int
    arrival: float = 0.0
    control_steps: int = 100
    substeps: int = 8


def poisson_requests(n: int, rate: float, seed: int, side_lo: int = 64, side_hi: int = 192, round_to: int = 32,
                     control_steps: int = 100, substeps: int = 8) -> List[Request]:
    """n requests with exponential inter-arrival times (rate per second) and cubic sides drawn
    log-uniform in [side_lo, side_hi], rounded to a multiple of ``round_to`` (the TMA kernel's
    tile: 16 in y, 32 in z)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    sides = np.exp(rng.uniform(math.log(side_lo), math.log(side_hi), n))
    sides = np.clip(np.round(sides / round_to) * round_to, side_lo, side_hi).astype(int)
    return [Request(i, int(sides[i]), int(rng.integers(1 << 30)), float(t[i]), control_steps, substeps)
            for i in range(n)]


def domain_bytes(side: int, storage: str) -> int:
    """Device bytes a resident domain holds: two moment buffers plus the per-solid state."""
    bpc = {"float32": 40, "float16": 20, "bfloat16": 20, "float64": 80}[storage]
    return 2 * side ** 3 * bpc + (1 << 20)


# ----------------------------------------------------------------------------- one domain
class Domain:
    """A resident request: its solver (one world), swimmer, pose and load buffers, stream and
    the CUDA graphs of its work (``batched``: the pose update of substep 0 and, per substep k,
    what follows the batched stream-collide; otherwise one graph of the whole control step)."""

    def __init__(self, req: Request, storage: str, vis: float, device, use_graph: bool = True,
                 batched: bool = False):
        if req.substeps < 2 or req.substeps % 2:
            # every control step starts from buffer 0: an even number of substeps ends there
            raise ValueError(f"request {req.rid}: substeps must be even and positive, got {req.substeps}")
        self.req = req
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        self.done = 0
        self.latencies: List[float] = []
        self.loads: List[np.ndarray] = []
        n = req.side
        with torch.cuda.stream(self.stream):
            self.solver = LBM_Solver3D(n, n, n, solid_num=SEGMENTS, storage=storage, device=device, use_graph=False,
                                       u_scale=0.02, s_scale=4e-4, with_flag=False, with_force=False)
            self.solver.set_viscosity(vis)
            self.swimmer = Swimmer.make(n, np.random.default_rng(req.seed))
            pos, quat = self.swimmer.poses(0.0)
            for k, mesh in enumerate(self.swimmer.meshes):
                self.solver.create_solid_from_mesh(k, mesh, lbm_position=tuple(pos[k]), lbm_scale=1.0 / n,
                                                   init_quaternion=tuple(quat[k]))
            S, dev = req.substeps, device
            # poses of every substep of a control step: positions and quaternions (w, x, y, z);
            # two pinned host copies so the next step's poses are written while the device
            # still reads the current ones
            self.pos_host = [torch.zeros((S, SEGMENTS, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
            self.quat_host = [torch.zeros((S, SEGMENTS, 4), dtype=torch.float32).pin_memory() for _ in range(2)]
            self.pos_dev = torch.zeros((S, SEGMENTS, 3), dtype=torch.float32, device=dev)
            self.quat_dev = torch.zeros((S, SEGMENTS, 4), dtype=torch.float32, device=dev)
            self.buf = 0
            # loads of every substep, written by the cut-link pass itself: [substep][force, torque][segment][3]
            self.loads_dev = torch.zeros((S, 2, SEGMENTS, 3), dtype=torch.float32, device=dev)
            self.loads_host = torch.zeros((S, 2, SEGMENTS, 3), dtype=torch.float32).pin_memory()
            self.ids = torch.arange(SEGMENTS, dtype=torch.int32, device=dev)
            self.zeros3 = torch.zeros((SEGMENTS, 3), dtype=torch.float32, device=dev)
            self.ones = torch.ones(SEGMENTS, dtype=torch.float32, device=dev)
        self.batched = bool(batched)
        self.graph = None
        self.pre_graph = None
        self.post_graphs: List[torch.cuda.CUDAGraph] = []
        if use_graph:
            self.stream.synchronize()
            if self.batched:
                self.pre_graph = self._capture(lambda: self._pose(0))
                S = req.substeps
                # what follows the batched stream-collide, cut links and boundaries of substep k:
                # the pose of substep k + 1 (nothing after the last substep)
                self.post_graphs = [self._capture(lambda k=k: self._pose(k + 1)) if k + 1 < S else None
                                    for k in range(S)]
            else:
                self.graph = self._capture(self._control_step)
        self.event = torch.cuda.Event()
        self.ready = torch.cuda.Event()  # batched: the domain's part of the current substep is done

    def _capture(self, fn) -> torch.cuda.CUDAGraph:
        g = torch.cuda.CUDAGraph()
        with _graph_capture(g, self.stream):
            fn()
        return g

    def _pose(self, k: int) -> None:
        """The swimmer's pose of substep k from the pose buffer (convert_and_update_solid_batch_3d)."""
        s = self.solver
        _lib.check(_lib.lib().hl_couple3d_update_solids(
            1, SEGMENTS, SEGMENTS, _lib.ptr(self.ids), self.pos_dev[k].data_ptr(), self.quat_dev[k].data_ptr(),
            _lib.ptr(self.zeros3), _lib.ptr(self.zeros3), _lib.ptr(self.ones),
            _lib.ptr(s.solid_position_all), _lib.ptr(s.solid_quaternion_all), _lib.ptr(s.mesh_transforms_all),
            _lib.ptr(s.mesh_transforms_last_all), _lib.ptr(s.mesh_transforms_initialized_all), _lib.stream_ptr()),
            "pose update")

    def _loads_out(self, k: int):
        return [(self.loads_dev[k, 0].data_ptr(), self.loads_dev[k, 1].data_ptr())]

    def _after_stream_collide(self, k: int, next_pose: bool) -> None:
        """Substep k after its stream-collide: cut links (loads into slot k), boundaries, and the
        pose of substep k + 1."""
        self.solver._launch(k % 2, _lib.stream_ptr(), loads_out=self._loads_out(k), stream_collide=False)
        if next_pose:
            self._pose(k + 1)


    def _control_step(self) -> None:
        """One control step on the current stream: per substep, the swimmer's pose and one LBM
        step with the cut links, whose loads go straight to the substep's slot of the load
        buffer."""
        for k in range(self.req.substeps):
            self._pose(k)
            self.solver._launch(k % 2, _lib.stream_ptr(), loads_out=self._loads_out(k))

    def stage_poses(self, step: int) -> None:
        """Host: the swimmer's poses for every substep of control step ``step``, into the host
        buffer that the launch of that step uploads."""
        S = self.req.substeps
        buf = step % 2
        pos, quat = self.swimmer.poses_at(np.arange(step * S + 1, step * S + S + 1))
        self.pos_host[buf].numpy()[...] = pos
        self.quat_host[buf].numpy()[...] = quat

    def launch(self) -> None:
        """Enqueue the next control step on the domain's stream (pose upload, the step, the
        load download)."""
        buf = self.done % 2
        with torch.cuda.stream(self.stream):
            self.pos_dev.copy_(self.pos_host[buf], non_blocking=True)
            self.quat_dev.copy_(self.quat_host[buf], non_blocking=True)
            if self.graph is not None:
                self.graph.replay()
            else:
                self._control_step()
            self.loads_host.copy_(self.loads_dev, non_blocking=True)
            self.event.record(self.stream)

    # batched: the engine interleaves these with the batched stream-collide of each substep
    def begin(self) -> None:
        """Pose upload and the pose of substep 0; records ``ready``."""
        buf = self.done % 2
        with torch.cuda.stream(self.stream):
            self.pos_dev.copy_(self.pos_host[buf], non_blocking=True)
            self.quat_dev.copy_(self.quat_host[buf], non_blocking=True)
            self.pre_graph.replay()
            self.ready.record(self.stream)

    def after(self, k: int, stream_collide_done: torch.cuda.Event) -> None:
        """Substep k's part after the batched stream-collide, cut links and boundaries (which
        ``stream_collide_done`` marks): the pose of substep k + 1; records ``ready``."""
        self.stream.wait_event(stream_collide_done)
        with torch.cuda.stream(self.stream):
            if self.post_graphs[k] is not None:
                self.post_graphs[k].replay()
            self.ready.record(self.stream)

    def end(self) -> None:
        """The load download; records ``event``."""
        with torch.cuda.stream(self.stream):
            self.loads_host.copy_(self.loads_dev, non_blocking=True)
            self.event.record(self.stream)

    def finish(self, latency: float) -> None:
        # per substep and segment: force then torque (the plain baseline's layout)
        self.loads.append(np.concatenate([self.loads_host[:, 0].numpy(), self.loads_host[:, 1].numpy()], axis=2))
        self.latencies.append(latency)
        self.done += 1

    @property
    def finished(self) -> bool:
        return self.done >= self.req.control_steps

    def release(self) -> None:
        self.graph = None
        self.pre_graph = None
        self.post_graphs = []
        self.solver = None


class BatchStep:
    """The batched stream-collide of a set of domains (hl_d3q27_stream_collide_batch): the
    descriptors (buffers, sizes, tensor maps of every domain) are written once for the set;
    each substep is then one launch at that substep's parity."""

    def __init__(self, domains: List["Domain"], stream: torch.cuda.Stream):
        L = _lib.lib()
        if len({d.req.substeps for d in domains}) != 1:
            raise ValueError("batched stream-collide: the domains need one number of substeps")
        flows = [d.solver.flows[0] for d in domains]
        vis = {float(f.vis_shear) for f in flows}
        if len(vis) != 1:
            raise ValueError("batched stream-collide: the domains need one viscosity")
        self.vis = vis.pop()
        self.n = len(flows)
        worlds = (_lib.hl_world3d * self.n)(*[f.world_struct(0) for f in flows])
        self.storage = worlds[0].storage
        nbytes = int(L.hl_d3q27_batch_bytes(self.n))
        dev = flows[0].device
        self.buf = torch.empty(nbytes + 64, dtype=torch.uint8, device=dev)
        self.ptr = (self.buf.data_ptr() + 63) // 64 * 64
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        n_items = ctypes.c_int(0)
        _lib.check(L.hl_d3q27_batch_prepare(worlds, self.n, self.ptr, nbytes, ctypes.byref(n_items),
                                            _lib.stream_ptr(stream)), "batched stream-collide (prepare)")
        self.n_items = int(n_items.value)

    def launch(self, parity: int, stream: torch.cuda.Stream) -> None:
        _lib.check(_lib.lib().hl_d3q27_stream_collide_batch(
            self.ptr, self.n, self.n_items, self.vis, ctypes.byref(self.storage), int(parity),
            self.status.data_ptr(), _lib.stream_ptr(stream)), "batched stream-collide")


class LinkBatch:
    """The cut links of a set of domains in one classify and one process launch
    (hl_d3q27_solid_links_batch). Each substep writes its loads into its own slot of every
    domain's load buffer, so there is one descriptor set per substep."""

    def __init__(self, domains: List[Domain], stream: torch.cuda.Stream):
        L = _lib.lib()
        flows = [d.solver.flows[0] for d in domains]
        self.vis = float(flows[0].vis_shear)
        self.n = len(domains)
        total = sum(int(d.solver.solid_num) for d in domains)
        nbytes = int(L.hl_d3q27_links_batch_bytes(self.n, total))
        dev = flows[0].device
        self.descs = []
        need = 0
        for k in range(domains[0].req.substeps):
            worlds = (_lib.hl_world3d * self.n)(*[f.world_struct(0) for f in flows])
            structs = []
            for d in domains:
                sst = d.solver._solids_struct(0)
                sst.force, sst.torque = d._loads_out(k)[0]
                structs.append(sst)
            solids = (_lib.hl_solids3d * self.n)(*structs)
            buf = torch.empty(nbytes + 64, dtype=torch.uint8, device=dev)
            ptr = (buf.data_ptr() + 63) // 64 * 64
            wi = ctypes.c_size_t(0)
            _lib.check(L.hl_d3q27_links_batch_prepare(worlds, solids, self.n, self.vis, ptr, nbytes, ctypes.byref(wi),
                                                      _lib.stream_ptr(stream)), "batched cut links (prepare)")
            self.descs.append((buf, ptr))
            need = max(need, int(wi.value))
        self.work = torch.zeros(max(need, 1), dtype=torch.int32, device=dev)

    def launch(self, k: int, stream: torch.cuda.Stream) -> None:
        """The cut links of substep k (parity k % 2), loads into slot k."""
        _lib.check(_lib.lib().hl_d3q27_solid_links_batch(
            self.descs[k][1], self.n, k % 2, self.work.data_ptr(), self.work.numel(), _lib.stream_ptr(stream)),
            "batched cut links")


class BcBatch:
    """The boundaries of a set of domains as three launches, one per wave, over all of them
    (hl_d3q27_apply_bc_batch) instead of three per domain. The descriptors cover both
    parities; each domain keeps its own boundary scratch."""

    def __init__(self, domains: List[Domain], stream: torch.cuda.Stream):
        L = _lib.lib()
        flows = [d.solver.flows[0] for d in domains]
        self.n = len(domains)
        nbytes = int(L.hl_d3q27_bc_batch_bytes(self.n))
        worlds = (_lib.hl_world3d * self.n)(*[f.world_struct(0) for f in flows])
        bcs = (_lib.hl_bc3d * self.n)(*[f.bc_struct() for f in flows])
        scratch = (ctypes.c_void_p * self.n)(*[_lib.ptr(d.solver._bc_scratch[0]) for d in domains])
        self.buf = torch.empty(nbytes + 16, dtype=torch.uint8, device=flows[0].device)
        self.ptr = (self.buf.data_ptr() + 15) // 16 * 16
        _lib.check(L.hl_d3q27_bc_batch_prepare(worlds, bcs, scratch, self.n, self.ptr, nbytes, _lib.stream_ptr(stream)),
                   "batched boundaries (prepare)")

    def launch(self, parity: int, stream: torch.cuda.Stream) -> None:
        _lib.check(_lib.lib().hl_d3q27_apply_bc_batch(self.ptr, self.n, int(parity), _lib.stream_ptr(stream)),
                   "batched boundaries")


class TickGraph:
    """One control step of a fixed set of batched domains as ONE CUDA graph: the pose of
    substep 0 of every domain, then per substep the batched stream-collide, cut links and
    boundaries (the cut links and boundaries per domain when ``links`` is None) followed by
    every domain's next pose, each domain on its own branch.
    Replaying it costs the host one launch instead of a few calls per domain and substep (which
    leave the device idle between substeps). The pose upload and load download stay outside, on
    the replaying stream."""

    def __init__(self, domains: List[Domain], batch: "BatchStep", main: torch.cuda.Stream,
                 links: Optional[LinkBatch] = None, bcs: Optional[BcBatch] = None):
        if (links is None) != (bcs is None):
            raise ValueError("TickGraph: batched cut links and batched boundaries go together")
        S = domains[0].req.substeps
        torch.cuda.synchronize()
        fork = torch.cuda.Event()
        sc_done = [torch.cuda.Event() for _ in range(S)]
        ready = [[torch.cuda.Event() for _ in range(S + 1)] for _ in domains]
        self.graph = torch.cuda.CUDAGraph()
        with _graph_capture(self.graph, main):
            fork.record(main)
            for d, rd in zip(domains, ready):
                d.stream.wait_event(fork)
                with torch.cuda.stream(d.stream):
                    d._pose(0)
                rd[0].record(d.stream)
            for k in range(S):
                for rd in ready:
                    main.wait_event(rd[k])
                batch.launch(k % 2, main)
                if links is not None:
                    links.launch(k, main)
                    bcs.launch(k % 2, main)
                sc_done[k].record(main)
                for d, rd in zip(domains, ready):
                    d.stream.wait_event(sc_done[k])
                    with torch.cuda.stream(d.stream):
                        if links is None:
                            d._after_stream_collide(k, k + 1 < S)
                        elif k + 1 < S:
                            d._pose(k + 1)
                    rd[k + 1].record(d.stream)
            for rd in ready:
                main.wait_event(rd[S])


# ----------------------------------------------------------------------------- engines
@dataclass
class ServeStats:
    env_steps: int
    wall_s: float
    latencies_s: List[float]
    results: Dict[int, np.ndarray]
    max_active: int
    admitted_order: List[int]
    fields: Dict[int, np.ndarray] = field(default_factory=dict)

    @property
    def env_steps_per_s(self) -> float:
        return self.env_steps / self.wall_s

    def pct(self, q: float) -> float:
        return float(np.percentile(np.array(self.latencies_s), q))


class ServeEngine:
    """Continuous batching of resident domains (see the module docstring)."""

    def __init__(self, storage: str = "float16", budget_bytes: float = 150e9, max_active: int = 32,
                 vis: float = 0.01, device=None, keep_fields: bool = False, batched: bool = False,
                 x_chunks: Optional[int] = None, link_blocks: Optional[int] = None):
        self.storage = storage
        self.budget = float(budget_bytes)
        self.max_active = int(max_active)
        self.vis = float(vis)
        self.device = _lib.require_cuda(device)
        self.keep_fields = bool(keep_fields)
        # per-domain graphs unless asked (see the module docstring); the batched stream-collide
        # takes float32/16 and bfloat16 storage only
        self.batched = bool(batched) and storage != "float64"
        # x chunks per tile column of the domains' stream-collide (the library's "d3q27_chunks"
        # while run() lasts; 0 keeps the library's choice). None: 1 for per-domain graphs, 0
        # for the batched form. The automatic split of a lone launch is sized to fill every SM
        # with one domain (a 64^3 domain gets chunks of 4 planes, each reading 2 halo planes
        # and refilling the copy pipeline); resident domains on their own streams fill the GPU
        # together, so whole columns spend less on halos and fills. The batched launch is the
        # opposite case: its items of 64-192 planes would end on the longest ones, so it keeps
        # its own ~32-plane chunks.
        if x_chunks is None:
            x_chunks = 0 if self.batched else 1
        self.x_chunks = int(x_chunks)
        if self.x_chunks < 0:
            raise ValueError(f"x_chunks must be >= 0, got {x_chunks}")
        # blocks of each domain's cut-link kernel (the library's "d3q27_link_blocks" while run()
        # lasts; 0 keeps the library's automatic grid). None: a quarter of the SM count for
        # per-domain graphs (16-warp blocks: 592 warps on a 148-SM B200), 0 for the batched form:
        # with resident domains sharing the GPU, fewer blocks per domain leave the other domains'
        # kernels room.
        if link_blocks is None:
            sms = torch.cuda.get_device_properties(self.device).multi_processor_count
            link_blocks = 0 if self.batched else max(1, sms // 4)
        self.link_blocks = int(link_blocks)
        if not 0 <= self.link_blocks <= 4096:
            raise ValueError(f"link_blocks must be in 0..4096, got {link_blocks}")

    def run(self, requests: List[Request], realtime: bool = True) -> ServeStats:
        """Serve the requests (arrival times honoured when ``realtime``) until all finish."""
        prev = {k: _lib.get_tuning(k) for k in ("d3q27_chunks", "d3q27_link_blocks")}
        _lib.set_tuning("d3q27_chunks", self.x_chunks)
        _lib.set_tuning("d3q27_link_blocks", self.link_blocks)
        try:
            return self._run(requests, realtime)
        finally:
            for k, v in prev.items():
                _lib.set_tuning(k, v)

    def _run(self, requests: List[Request], realtime: bool) -> ServeStats:
        pending = sorted(requests, key=lambda r: r.arrival)
        active: List[Domain] = []
        used = 0.0
        lat, results, order, fields = [], {}, [], {}
        peak = 0
        steps = 0
        t_start = time.perf_counter()

        def now():
            return time.perf_counter() - t_start

        prepared: List[Domain] = []  # admitted, built while the device ran a tick, not yet stepped

        def build(limit: int) -> List[Domain]:
            """Domains for up to ``limit`` pending requests (arrived, within the HBM budget)."""
            nonlocal used
            out = []
            while len(out) < limit and pending and (not realtime or pending[0].arrival <= now()):
                need = domain_bytes(pending[0].side, self.storage)
                if used + need > self.budget:
                    break
                r = pending.pop(0)
                d = Domain(r, self.storage, self.vis, self.device, batched=self.batched)
                d.stage_poses(0)
                out.append(d)
                used += need
                order.append(r.rid)
            return out

        def admit():
            while prepared and len(active) < self.max_active:
                active.append(prepared.pop(0))
            active.extend(build(self.max_active - len(active)))

        main = torch.cuda.Stream(device=self.device)
        sc_done = torch.cuda.Event()
        tick_done = torch.cuda.Event()
        batch, links, bcs, batch_ids, tick_graph, stable = None, None, None, None, None, 0
        while pending or active or prepared:
            admit()
            if not active:
                time.sleep(max(0.0, min(pending[0].arrival - now(), 0.01)))
                continue
            peak = max(peak, len(active))
            running = list(active)
            if self.batched:
                if batch_ids != [id(d) for d in running]:
                    batch = BatchStep(running, main)  # the set changed: new descriptors
                    links = LinkBatch(running, main)
                    bcs = BcBatch(running, main)
                    batch_ids = [id(d) for d in running]
                    tick_graph, stable = None, 0
                else:
                    stable += 1
                # one graph per set, once the set has held for two ticks (while domains arrive
                # or finish every tick, capturing would cost more than it saves)
                if tick_graph is None and stable >= 2:
                    tick_graph = TickGraph(running, batch, main, links, bcs)
            t0 = time.perf_counter()
            if tick_graph is not None:
                with torch.cuda.stream(main):
                    for d in running:
                        buf = d.done % 2
                        d.pos_dev.copy_(d.pos_host[buf], non_blocking=True)
                        d.quat_dev.copy_(d.quat_host[buf], non_blocking=True)
                    tick_graph.graph.replay()
                    for d in running:
                        d.loads_host.copy_(d.loads_dev, non_blocking=True)
                    tick_done.record(main)
            elif self.batched:
                for d in running:
                    d.begin()
                for k in range(running[0].req.substeps):
                    for d in running:
                        main.wait_event(d.ready)
                    batch.launch(k % 2, main)
                    links.launch(k, main)
                    bcs.launch(k % 2, main)
                    sc_done.record(main)
                    for d in running:
                        d.after(k, sc_done)
                for d in running:
                    d.end()
            else:
                for d in running:
                    d.launch()
            # while the device works: the poses of every domain's next control step, and the
            # domains of the requests that take the slots freed after this tick (a domain costs
            # ~8 ms of host time to build, which otherwise leaves the device idle), one at a time
            # and only while the tick is still running, so that the tick's latency stays its own
            for d in running:
                if d.done + 1 < d.req.control_steps:
                    d.stage_poses(d.done + 1)
            want = self.max_active - len(active) + sum(1 for d in running if d.done + 1 >= d.req.control_steps)
            while len(prepared) < want and not (tick_done.query() if tick_graph is not None
                                                else all(d.event.query() for d in running)):
                got = build(1)
                if not got:
                    break
                prepared.extend(got)
            if tick_graph is not None:
                tick_done.synchronize()
            else:
                for d in running:
                    d.event.synchronize()
            t1 = time.perf_counter()
            for d in running:
                d.finish(t1 - t0)
                lat.append(t1 - t0)
                steps += 1
            for d in [d for d in active if d.finished]:
                active.remove(d)
                results[d.req.rid] = np.stack(d.loads)
                if self.keep_fields:  # the final velocity field, for accuracy checks
                    fields[d.req.rid] = d.solver.flows[0].decoded()[1:4].double().cpu().numpy()
                used -= domain_bytes(d.req.side, self.storage)
                d.release()
        torch.cuda.synchronize()
        return ServeStats(steps, time.perf_counter() - t_start, lat, results, peak, order, fields)


def run_plain(requests: List[Request], storage: str = "float32", vis: float = 0.01, device=None) -> ServeStats:
    """Baseline: one request at a time through the plain solver (LBM_Solver3D.step, one graph
    launch per LBM step), poses through the coupling kernel, loads read back every control
    step; requests in arrival order, each started when it has arrived and the previous one
    finished."""
    device = _lib.require_cuda(device)
    lat, results, order = [], {}, []
    steps = 0
    t_start = time.perf_counter()
    for r in sorted(requests, key=lambda r: r.arrival):
        wait = r.arrival - (time.perf_counter() - t_start)
        if wait > 0:
            time.sleep(wait)
        d = PlainDomain(r, storage, vis, device)
        for _ in range(r.control_steps):
            t0 = time.perf_counter()
            d.control_step()
            lat.append(time.perf_counter() - t0)
            steps += 1
        results[r.rid] = np.stack(d.loads)
        order.append(r.rid)
    torch.cuda.synchronize()
    return ServeStats(steps, time.perf_counter() - t_start, lat, results, 1, order)


class PlainDomain:
    """A request on the plain solver: LBM_Solver3D.step() per substep (its own CUDA graph)."""

    def __init__(self, req: Request, storage: str, vis: float, device):
        n = req.side
        self.req = req
        self.solver = LBM_Solver3D(n, n, n, solid_num=SEGMENTS, storage=storage, device=device, u_scale=0.02,
                                   s_scale=4e-4, with_flag=False, with_force=False)
        self.solver.set_viscosity(vis)
        self.swimmer = Swimmer.make(n, np.random.default_rng(req.seed))
        pos, quat = self.swimmer.poses(0.0)
        for k, mesh in enumerate(self.swimmer.meshes):
            self.solver.create_solid_from_mesh(k, mesh, lbm_position=tuple(pos[k]), lbm_scale=1.0 / n,
                                               init_quaternion=tuple(quat[k]))
        self.done = 0
        self.loads: List[np.ndarray] = []
        dev = device
        self.ids = torch.arange(SEGMENTS, dtype=torch.int32, device=dev)
        self.zeros3 = torch.zeros((SEGMENTS, 3), dtype=torch.float32, device=dev)
        self.ones = torch.ones(SEGMENTS, dtype=torch.float32, device=dev)
        S = req.substeps
        self.pos_host = torch.zeros((S, 1, SEGMENTS, 3), dtype=torch.float32).pin_memory()
        self.quat_host = torch.zeros((S, 1, SEGMENTS, 4), dtype=torch.float32).pin_memory()
        self.pos_dev = torch.zeros((S, 1, SEGMENTS, 3), dtype=torch.float32, device=dev)
        self.quat_dev = torch.zeros((S, 1, SEGMENTS, 4), dtype=torch.float32, device=dev)
        self.loads_dev = torch.zeros((req.substeps, SEGMENTS, 6), dtype=torch.float32, device=dev)

    def control_step(self) -> None:
        from . import coupling

        s, S = self.solver, self.req.substeps
        t0 = self.done * S
        pos, quat = self.swimmer.poses_at(np.arange(t0 + 1, t0 + S + 1))
        self.pos_host.numpy()[:, 0] = pos
        self.quat_host.numpy()[:, 0] = quat
        self.pos_dev.copy_(self.pos_host, non_blocking=True)
        self.quat_dev.copy_(self.quat_host, non_blocking=True)
        f = s.flows[0]
        for k in range(S):
            coupling.convert_and_update_solid_batch_3d(s, self.ids, self.pos_dev[k], self.quat_dev[k], self.zeros3,
                                                       self.zeros3, self.ones)
            s.step()
            self.loads_dev[k, :, :3].copy_(f.solid_force)
            self.loads_dev[k, :, 3:].copy_(f.solid_torque)
        self.loads.append(self.loads_dev.cpu().numpy())
        self.done += 1
