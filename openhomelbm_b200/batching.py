"""Batching form: D2Q9 worlds of different sizes stepped together by one persistent launch.

``WorldBatch2D`` holds uneven worlds (each a ``HomeFlow`` with its own polygon solids), their
descriptor array on the device and a tile work-list over all of them. One step is
``hl_d2q9_step_tiles``: the segment transforms of every world, the stream phase as a single
persistent launch whose CTAs take the tiles of the list in turn, the cut-link band and the
boundaries. The tile shape and the number of persistent CTAs (the work-list granularity) are
chosen by ``TileAutotuner``, which times every supported combination on the batch itself and
caches the winner per batch signature.

``SwimmerBatch2D`` is the batching workload: worlds whose sides are drawn log-uniform from a
seed, each holding a chain of capsules (polygon solids) that follows a prescribed travelling
wave, stepped ``substeps`` LBM steps per control step with the per-capsule force and torque of
every substep returned. A control step (the pose updates of all worlds through the 2D coupling
kernel, the substeps, the load copies) is captured as one CUDA graph for the admitted set.
``run_sequential_plain`` is its baseline: the same worlds one at a time through the plain
``LBM_Solver`` (float32 storage, one graph launch per LBM step).

The reference batches only same-size worlds (LBM_Solver's nworld, envs/lbm/lbm_solver.py:
117-139) with one launch per world-sized grid; the tile kernel's arithmetic is that of the
plain stream phase, so every world's result is identical to stepping it alone.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .lbm.lbm_core import HomeFlow

# ----------------------------------------------------------------------------- tile lists


def tile_shapes() -> List[Tuple[int, int]]:
    """The tile shapes (cells along x, along y) the persistent stream launch supports."""
    L = _lib.lib()
    n = int(L.hl_d2q9_tile_shapes(None, 0))
    out = np.zeros(2 * n, np.int32)
    L.hl_d2q9_tile_shapes(out.ctypes.data, n)
    return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(n)]


def tile_list(nx: Sequence[int], ny: Sequence[int], tile: Tuple[int, int]) -> np.ndarray:
    """The tile work-list of worlds nx[w] x ny[w]: (n_tiles, 4) int32 rows (world, x0, y0, 0),
    world-major, x outer, y inner."""
    L = _lib.lib()
    nx_a = np.ascontiguousarray(nx, np.int32)
    ny_a = np.ascontiguousarray(ny, np.int32)
    count = ctypes.c_size_t(0)
    _lib.check(L.hl_d2q9_tile_list(nx_a.ctypes.data, ny_a.ctypes.data, len(nx_a), int(tile[0]), int(tile[1]), None, 0,
                                   ctypes.byref(count)), "tile list")
    out = np.zeros((int(count.value), 4), np.int32)
    _lib.check(L.hl_d2q9_tile_list(nx_a.ctypes.data, ny_a.ctypes.data, len(nx_a), int(tile[0]), int(tile[1]),
                                   out.ctypes.data, out.shape[0], ctypes.byref(count)), "tile list")
    return out


@dataclass(frozen=True)
class TileConfig:
    """A launch configuration of the persistent stream phase."""

    tile_x: int
    tile_y: int
    ctas: int  # persistent CTAs (the grid), at most one per tile


# ----------------------------------------------------------------------------- batch of worlds
class WorldBatch2D:
    """Uneven D2Q9 worlds stepped by ``hl_d2q9_step_tiles``. All worlds share the storage type
    and are stepped together (one parity)."""

    def __init__(self, flows: Sequence[HomeFlow], device=None):
        if not flows:
            raise ValueError("WorldBatch2D needs at least one world")
        codes = {f.storage_code for f in flows}
        if len(codes) != 1:
            raise ValueError("all worlds of a batch must use the same storage type")
        self.flows = list(flows)
        self.n = len(self.flows)
        self.device = _lib.require_cuda(device if device is not None else self.flows[0].device)
        self.storage_code = codes.pop()
        L = _lib.lib()
        self._desc_bytes = int(L.hl_d2q9_desc_bytes())
        self.desc = torch.zeros(self._desc_bytes * self.n, dtype=torch.uint8, device=self.device)
        self._tiles: Dict[Tuple[int, int], torch.Tensor] = {}
        self.config: Optional[TileConfig] = None
        self.any_solid = False
        self.upload()

    @property
    def parity(self) -> int:
        return self.flows[0].parity

    def signature(self) -> Tuple:
        """What the autotuner's choice depends on: the worlds' sizes and the storage type."""
        return (self.storage_code, tuple((f.nx, f.ny, bool(f.periodic)) for f in self.flows))

    def cells(self) -> int:
        return sum(f.nx * f.ny for f in self.flows)

    def upload(self) -> None:
        """Pack every world's descriptor (buffers, viscosity, boundaries, solids) to the device.
        Call again after changing a world's parameters; a captured graph stays valid (it bakes
        only the descriptor array's address)."""
        L = _lib.lib()
        host = bytearray(self._desc_bytes * self.n)
        base = (ctypes.c_char * len(host)).from_buffer(host)
        any_solid = False
        for k, f in enumerate(self.flows):
            s = f.solids_struct()
            any_solid |= s is not None
            _lib.check(L.hl_d2q9_pack(f.world_struct(), f.step_struct(), f.bc_struct(), s,
                                      ctypes.addressof(base) + k * self._desc_bytes), "pack world")
        self.desc.copy_(torch.frombuffer(host, dtype=torch.uint8))
        self.any_solid = any_solid

    def tiles(self, shape: Tuple[int, int]) -> torch.Tensor:
        """The device tile list for a tile shape (built once per shape)."""
        t = self._tiles.get(shape)
        if t is None:
            host = tile_list([f.nx for f in self.flows], [f.ny for f in self.flows], shape)
            t = torch.tensor(host, dtype=torch.int32, device=self.device)
            self._tiles[shape] = t
        return t

    def launch(self, parity: int, stream, config: Optional[TileConfig] = None, phases: int = _lib.HL_PHASE_ALL,
               any_solid: Optional[bool] = None) -> None:
        """Enqueue one step of every world (no swap) on ``stream``."""
        cfg = config or self.config
        if cfg is None:
            raise RuntimeError("WorldBatch2D: no launch configuration (run TileAutotuner.tune first)")
        tl = self.tiles((cfg.tile_x, cfg.tile_y))
        solid = self.any_solid if any_solid is None else any_solid
        _lib.check(_lib.lib().hl_d2q9_step_tiles(_lib.ptr(self.desc), self.n, parity, self.storage_code, _lib.ptr(tl),
                                                 tl.shape[0], cfg.tile_x, cfg.tile_y, cfg.ctas, int(solid), phases,
                                                 stream), "WorldBatch2D.step")

    def step(self) -> None:
        """One step of every world on the current stream (eager), then the buffer swap."""
        self.launch(self.parity, _lib.stream_ptr())
        for f in self.flows:
            f.swap()


# ----------------------------------------------------------------------------- autotuner
class TileAutotuner:
    """Chooses the tile shape and the persistent grid of a batch by timing every supported tile
    shape with ``ctas_per_sm`` CTAs per SM on the batch's own worlds (stream phase only, CUDA
    events, median of ``reps`` launches after ``warmup``). The stream phase writes only the
    worlds' post buffers, which the next step overwrites, so tuning leaves the state as it
    was. Results are cached per batch signature; ``table`` keeps every timing."""

    def __init__(self, ctas_per_sm: Sequence[int] = (1, 2, 4, 8), reps: int = 5, warmup: int = 2):
        self.ctas_per_sm = tuple(int(c) for c in ctas_per_sm)
        self.reps, self.warmup = int(reps), int(warmup)
        self.cache: Dict[Tuple, TileConfig] = {}
        self.table: Dict[Tuple, Dict[TileConfig, float]] = {}

    def candidates(self, batch: WorldBatch2D) -> List[TileConfig]:
        sms = torch.cuda.get_device_properties(batch.device).multi_processor_count
        out = []
        for shape in tile_shapes():
            n_tiles = batch.tiles(shape).shape[0]
            seen = set()
            for c in self.ctas_per_sm:
                ctas = max(1, min(n_tiles, c * sms))
                if ctas not in seen:
                    seen.add(ctas)
                    out.append(TileConfig(shape[0], shape[1], ctas))
        return out

    def tune(self, batch: WorldBatch2D) -> TileConfig:
        key = batch.signature()
        hit = self.cache.get(key)
        if hit is not None:
            batch.config = hit
            return hit
        st = _lib.stream_ptr()
        times: Dict[TileConfig, float] = {}
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for cfg in self.candidates(batch):
            for _ in range(self.warmup):
                batch.launch(batch.parity, st, cfg, phases=_lib.HL_PHASE_STREAM, any_solid=False)
            samples = []
            for _ in range(self.reps):
                a.record()
                batch.launch(batch.parity, st, cfg, phases=_lib.HL_PHASE_STREAM, any_solid=False)
                b.record()
                b.synchronize()
                samples.append(a.elapsed_time(b))
            times[cfg] = float(np.median(samples))
        best = min(times, key=times.get)
        self.cache[key] = best
        self.table[key] = times
        batch.config = best
        return best


# ----------------------------------------------------------------------------- swimmer workload
def capsule_polygon(half_length: float, radius: float, n_arc: int = 13) -> np.ndarray:
    """Outline of a capsule (a stadium) centred at the origin along x: the segment
    [-half_length, half_length] widened by ``radius``; two semicircles of ``n_arc`` points,
    counter-clockwise, in lattice units."""
    pts = []
    for k in range(n_arc):  # right cap, -90 .. +90 degrees
        a = -math.pi / 2 + math.pi * k / (n_arc - 1)
        pts.append((half_length + radius * math.cos(a), radius * math.sin(a)))
    for k in range(n_arc):  # left cap, +90 .. +270 degrees
        a = math.pi / 2 + math.pi * k / (n_arc - 1)
        pts.append((-half_length + radius * math.cos(a), radius * math.sin(a)))
    return np.array(pts, np.float32)


@dataclass
class CapsuleChain:
    """A planar swimmer: ``n_capsules`` capsules along a body of length ``length`` whose
    centreline follows y(s, t) = A(s) sin(2 pi (s / lambda - f t)), A rising linearly from
    ``a_head`` L at the head (s = 0) to ``a_tail`` L at the tail, lambda = L. t counts control
    steps; ``freq`` is per control step. Capsule k spans s in [k L / n, (k + 1) L / n]; its pose
    is the midpoint of that chord and the chord's direction."""

    head: Tuple[float, float]
    freq: float
    length: float = 64.0
    n_capsules: int = 8
    radius: float = 4.0
    a_head: float = 0.02
    a_tail: float = 0.1

    def centreline(self, s: np.ndarray, t: np.ndarray) -> np.ndarray:
        L = self.length
        amp = L * (self.a_head + (self.a_tail - self.a_head) * s / L)
        return amp * np.sin(2 * np.pi * (s / L - self.freq * t))

    def poses_at(self, t: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        """Capsule centres (T, n, 2) and angles (T, n) at control-step times t (T,)."""
        t = np.asarray(t, np.float64)[:, None]
        s = np.linspace(0.0, self.length, self.n_capsules + 1)[None, :]
        y = self.centreline(s, t)
        x = np.broadcast_to(self.head[0] + s, y.shape)
        cx = 0.5 * (x[:, 1:] + x[:, :-1])
        cy = self.head[1] + 0.5 * (y[:, 1:] + y[:, :-1])
        ang = np.arctan2(y[:, 1:] - y[:, :-1], x[:, 1:] - x[:, :-1])
        return np.stack([cx, cy], axis=2), ang


def chain_poses(chains: Sequence[CapsuleChain], t: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """CapsuleChain.poses_at of many chains of the same geometry (length, capsules, amplitude
    envelope) at once: centres (T, W, n, 2) and angles (T, W, n)."""
    c0 = chains[0]
    L, n = c0.length, c0.n_capsules
    if any((c.length, c.n_capsules, c.a_head, c.a_tail) != (L, n, c0.a_head, c0.a_tail) for c in chains):
        raise ValueError("chain_poses: every chain must have the same geometry")
    t = np.asarray(t, np.float64)[:, None, None]
    f = np.array([c.freq for c in chains], np.float64)[None, :, None]
    hx = np.array([c.head[0] for c in chains], np.float64)[None, :, None]
    hy = np.array([c.head[1] for c in chains], np.float64)[None, :, None]
    s = np.linspace(0.0, L, n + 1)[None, None, :]
    amp = L * (c0.a_head + (c0.a_tail - c0.a_head) * s / L)
    y = amp * np.sin(2 * np.pi * (s / L - f * t))
    x = np.broadcast_to(hx + s, y.shape)
    cx = 0.5 * (x[..., 1:] + x[..., :-1])
    cy = hy + 0.5 * (y[..., 1:] + y[..., :-1])
    ang = np.arctan2(y[..., 1:] - y[..., :-1], x[..., 1:] - x[..., :-1])
    return np.stack([cx, cy], axis=-1), ang


def batch_sizes(n_worlds: int, seed: int, nx_range=(256, 1024), ny_range=(128, 512)) -> List[Tuple[int, int]]:
    """World sizes nx ~ logU(nx_range), ny ~ logU(ny_range), drawn independently from
    default_rng(seed) and rounded to integers."""
    rng = np.random.default_rng(seed)
    nx = np.rint(np.exp(rng.uniform(math.log(nx_range[0]), math.log(nx_range[1]), n_worlds))).astype(int)
    ny = np.rint(np.exp(rng.uniform(math.log(ny_range[0]), math.log(ny_range[1]), n_worlds))).astype(int)
    return [(int(a), int(b)) for a, b in zip(nx, ny)]


@dataclass
class SwimmerSpec:
    """One world of the workload: its size and its swimmer."""

    nx: int
    ny: int
    chain: CapsuleChain


def swimmer_specs(n_worlds: int = 64, seed: int = 0, freq_range=(0.002, 0.01)) -> List[SwimmerSpec]:
    """The worlds of the batching workload: sizes from ``batch_sizes``, then per world a
    frequency f ~ U(freq_range) per control step from the same generator; the head sits at
    (nx / 4, ny / 2)."""
    sizes = batch_sizes(n_worlds, seed)
    rng = np.random.default_rng(seed + 1)
    freqs = rng.uniform(freq_range[0], freq_range[1], n_worlds)
    return [SwimmerSpec(nx, ny, CapsuleChain(head=(0.25 * nx, 0.5 * ny), freq=float(f)))
            for (nx, ny), f in zip(sizes, freqs)]


def _new_world(spec: SwimmerSpec, storage: str, vis: float, device, flow_views=None) -> HomeFlow:
    f = HomeFlow()
    f.Initialize(spec.nx, spec.ny, n_objects=spec.chain.n_capsules, device=device, storage=storage, u_scale=0.02,
                 s_scale=4e-4)
    f.vis_shear = float(vis)
    if flow_views is not None:  # batched pose / load rows (the coupling kernels' layout)
        pos, ang, loads = flow_views
        f.solid_position, f.solid_angle = pos, ang
        f.solid_forcex, f.solid_forcey, f.torque = loads[0], loads[1], loads[2]
    L = _lib.lib()
    st = _lib.stream_ptr()
    _lib.check(L.hl_d2q9_init_boundary(f.nx, f.ny, _lib.ptr(f.flag), st), "InitBoundary")
    _lib.check(L.hl_d2q9_init_uniform(f.nx, f.ny, _lib.hl_storage(f.storage_code, f.u_scale, f.s_scale),
                                      _lib.ptr(f.moments[0]), _lib.ptr(f.moments[1]), _lib.ptr(f.force[0]),
                                      _lib.ptr(f.force[1]), 0.0, 0.0, st), "InitFlow")
    ch = spec.chain
    poly = capsule_polygon(0.5 * ch.length / ch.n_capsules, ch.radius)
    pos, ang = ch.poses_at(np.zeros(1))
    for k in range(ch.n_capsules):
        f.configure_solid(k, poly, (float(pos[0, k, 0]), float(pos[0, k, 1])), angle=float(ang[0, k]),
                          scale=1.0 / spec.nx)
    return f


def _yaw_quat(angle: np.ndarray) -> np.ndarray:
    """(w, x, y, z) quaternions of yaw rotations, the layout MuJoCo's xquat uses."""
    out = np.zeros(angle.shape + (4,), np.float32)
    out[..., 0] = np.cos(0.5 * angle)
    out[..., 3] = np.sin(0.5 * angle)
    return out


@dataclass
class BatchStats:
    control_steps: int
    substeps: int
    wall_s: float
    cell_updates: int
    latencies_s: List[float]
    loads: np.ndarray  # [control step][substep][world][3 (fx, fy, torque)][capsule]
    config: Optional[TileConfig] = None
    tune_table: Dict = field(default_factory=dict)

    @property
    def mlups(self) -> float:
        return self.cell_updates / self.wall_s / 1e6


class SwimmerBatch2D:
    """The batching workload on one GPU (see the module docstring)."""

    def __init__(self, specs: Sequence[SwimmerSpec], storage: str = "float16", substeps: int = 8, vis: float = 0.01,
                 device=None, autotuner: Optional[TileAutotuner] = None, use_graph: bool = True):
        self.specs = list(specs)
        self.W = len(self.specs)
        self.n = self.specs[0].chain.n_capsules
        if any(s.chain.n_capsules != self.n for s in self.specs):
            raise ValueError("every world of a batch must hold the same number of capsules")
        self.S = int(substeps)
        self.device = dev = _lib.require_cuda(device)
        f32 = dict(dtype=torch.float32, device=dev)
        W, n, S = self.W, self.n, self.S
        self.position_all = torch.zeros((W, n, 2), **f32)
        self.angle_all = torch.zeros((W, n), **f32)
        self.loads_all = torch.zeros((W, 3, n), **f32)
        self.flows = [_new_world(sp, storage, vis, dev, (self.position_all[w], self.angle_all[w], self.loads_all[w]))
                      for w, sp in enumerate(self.specs)]
        self.batch = WorldBatch2D(self.flows, dev)
        self.autotuner = autotuner or TileAutotuner()
        self.config = self.autotuner.tune(self.batch)
        self.ids = torch.arange(n, dtype=torch.int32, device=dev)
        self.zeros2 = torch.zeros((n, 2), **f32)
        self.ones = torch.ones(n, **f32)
        # two pinned pose buffers: the host writes the next control step's poses into one while
        # the device reads the other
        self.pos_host = [torch.zeros((S, W, n, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
        self.quat_host = [torch.zeros((S, W, n, 4), dtype=torch.float32).pin_memory() for _ in range(2)]
        self.event = torch.cuda.Event()
        self.pos_dev = torch.zeros((S, W, n, 3), **f32)
        self.quat_dev = torch.zeros((S, W, n, 4), **f32)
        self.loads_dev = torch.zeros((S, W, 3, n), **f32)
        self.loads_host = torch.zeros((S, W, 3, n), dtype=torch.float32).pin_memory()
        self.done = 0
        torch.cuda.synchronize()
        self.graph = None
        if use_graph:
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._control_step()
            torch.cuda.synchronize()

    def _control_step(self) -> None:
        L = _lib.lib()
        st = _lib.stream_ptr()
        W, n = self.W, self.n
        for k in range(self.S):
            _lib.check(L.hl_couple2d_update_solids(W, n, n, _lib.ptr(self.ids), _lib.ptr(self.pos_dev[k]),
                                                   _lib.ptr(self.quat_dev[k]), _lib.ptr(self.zeros2),
                                                   _lib.ptr(self.zeros2), _lib.ptr(self.ones),
                                                   _lib.ptr(self.position_all), _lib.ptr(self.angle_all), st),
                       "pose update")
            self.batch.launch(k % 2, st)
            self.loads_dev[k].copy_(self.loads_all)

    def stage_poses(self, step: int, buf: int = 0) -> None:
        """Host: every world's capsule poses for the substeps of control step ``step`` (time in
        control steps: substep k of step c is at c + (k + 1) / substeps), into pose buffer buf."""
        t = step + (np.arange(self.S) + 1.0) / self.S
        pos, ang = chain_poses([sp.chain for sp in self.specs], t)
        self.pos_host[buf].numpy()[..., :2] = pos
        self.quat_host[buf].numpy()[...] = _yaw_quat(ang)

    def _enqueue(self, buf: int) -> None:
        self.pos_dev.copy_(self.pos_host[buf], non_blocking=True)
        self.quat_dev.copy_(self.quat_host[buf], non_blocking=True)
        if self.graph is not None:
            self.graph.replay()
        else:
            self._control_step()
        self.loads_host.copy_(self.loads_dev, non_blocking=True)
        self.event.record()

    def control_step(self) -> np.ndarray:
        """Advance every world by one control step; returns the loads [substep][world][3][n]."""
        self.stage_poses(self.done, 0)
        self._enqueue(0)
        self.event.synchronize()
        self.done += 1
        return self.loads_host.numpy().copy()

    def run(self, control_steps: int) -> BatchStats:
        """``control_steps`` control steps; the poses of step c + 1 are computed on the host while
        the device runs step c. A control step's latency is from its enqueue to its loads."""
        lat, loads = [], []
        t0 = time.perf_counter()
        if control_steps > 0:
            self.stage_poses(self.done, 0)
        for c in range(control_steps):
            buf = c % 2
            a = time.perf_counter()
            self._enqueue(buf)
            if c + 1 < control_steps:
                self.stage_poses(self.done + 1, buf ^ 1)
            self.event.synchronize()
            loads.append(self.loads_host.numpy().copy())
            lat.append(time.perf_counter() - a)
            self.done += 1
        wall = time.perf_counter() - t0
        cells = self.batch.cells() * self.S * control_steps
        key = self.batch.signature()
        return BatchStats(control_steps, self.S, wall, cells, lat, np.stack(loads), self.config,
                          dict(self.autotuner.table.get(key, {})))


def run_sequential_plain(specs: Sequence[SwimmerSpec], control_steps: int, substeps: int = 8, vis: float = 0.01,
                         storage: str = "float32", device=None) -> BatchStats:
    """Baseline: the worlds one after another through the plain LBM_Solver (one graph launch
    per LBM step), poses through the 2D coupling kernel, loads read back every control step.
    The wall time is the stepping time of all worlds (each world's set-up excluded)."""
    from .lbm import LBM_Solver

    dev = _lib.require_cuda(device)
    L = _lib.lib()
    lat, per_world = [], []
    cells = 0
    wall = 0.0  # stepping time only: each world's set-up is outside it, as the batch's is
    for sp in specs:
        n = sp.chain.n_capsules
        s = LBM_Solver(sp.nx, sp.ny, solid_num=n, storage=storage, device=dev)
        f = s.flows[0]
        f.vis_shear = float(vis)
        poly = capsule_polygon(0.5 * sp.chain.length / n, sp.chain.radius)
        pos0, ang0 = sp.chain.poses_at(np.zeros(1))
        for k in range(n):
            f.configure_solid(k, poly, (float(pos0[0, k, 0]), float(pos0[0, k, 1])), angle=float(ang0[0, k]),
                              scale=1.0 / sp.nx)
        f32 = dict(dtype=torch.float32, device=dev)
        ids = torch.arange(n, dtype=torch.int32, device=dev)
        zeros2, ones = torch.zeros((n, 2), **f32), torch.ones(n, **f32)
        pos_host = torch.zeros((substeps, n, 3), dtype=torch.float32).pin_memory()
        quat_host = torch.zeros((substeps, n, 4), dtype=torch.float32).pin_memory()
        pos_dev = torch.zeros((substeps, n, 3), **f32)
        quat_dev = torch.zeros((substeps, n, 4), **f32)
        loads_dev = torch.zeros((substeps, 3, n), **f32)
        out = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for c in range(control_steps):
            a = time.perf_counter()
            pos, ang = sp.chain.poses_at(c + (np.arange(substeps) + 1.0) / substeps)
            pos_host.numpy()[:, :, :2] = pos
            quat_host.numpy()[...] = _yaw_quat(ang)
            pos_dev.copy_(pos_host, non_blocking=True)
            quat_dev.copy_(quat_host, non_blocking=True)
            st = _lib.stream_ptr()
            for k in range(substeps):
                _lib.check(L.hl_couple2d_update_solids(1, n, n, _lib.ptr(ids), _lib.ptr(pos_dev[k]),
                                                       _lib.ptr(quat_dev[k]), _lib.ptr(zeros2), _lib.ptr(zeros2),
                                                       _lib.ptr(ones), _lib.ptr(s.solid_position_all),
                                                       _lib.ptr(s.solid_angle_all), st), "pose update")
                s.step()
                loads_dev[k].copy_(s.solid_loads_all[0])
            out.append(loads_dev.cpu().numpy())
            lat.append(time.perf_counter() - a)
        torch.cuda.synchronize()
        wall += time.perf_counter() - t0
        per_world.append(np.stack(out))
        cells += sp.nx * sp.ny * substeps * control_steps
        del s
    # [control step][substep][world][3][n], the batch's layout
    loads = np.stack(per_world, axis=2)
    return BatchStats(control_steps, substeps, wall, cells, lat, loads)
