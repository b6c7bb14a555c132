"""Serving loop for scattering solves (FarField, FarField.hpp:28-144) on one GPU.

Requests -- a mesh, one wavenumber and 1-64 plane-wave directions -- arrive
while others are running.  The server keeps a pool of worker slots; each slot
owns one library context on its own CUDA stream, with its mesh, Krylov basis,
intermediate blocks and solution resident on the device, and runs one solve at
a time.  A request is admitted when a slot is free and its device-memory
footprint fits the budget (continuous batching: admission happens whenever a
running solve finishes, not in waves), so the solves of several requests
overlap on the GPU.  Inside a solve the operator apply runs in the context's
apply mode (the compensated tensor-core form by default, with the tile
settings picked by the library's autotuner) and the solver's inner operators
are replayed as CUDA graphs.

The admission logic (`Scheduler`) is independent of the GPU and is tested on
the CPU; `SolveServer` drives `Helmholtz_CUDA` contexts from worker threads
(the C ABI releases the Python GIL during each call).
"""
from __future__ import annotations

import collections
import dataclasses
import threading
import time
from typing import Callable, Optional

import numpy as np

# wave_chunk_size values the incident-wave path accepts (CreateIncidentWave.hpp:35-45,
# IncidentWaveKernel_Plane.hpp:15-182) that the tensor-core form runs as 16-column groups
RHS_SIZES = (16, 32, 64)


def padded_rhs(nrhs: int) -> int:
    """Right-hand-side count a request of `nrhs` directions is solved with."""
    for s in RHS_SIZES:
        if nrhs <= s:
            return s
    raise ValueError(f"at most {RHS_SIZES[-1]} right-hand sides per request, got {nrhs}")


def solve_footprint_bytes(nv: int, nt: int, wc: int, restart: int = 30) -> int:
    """Device memory a FarField solve of this size holds in a context: the
    GMRES basis ((restart + 1) vectors of nv x wc complex128), the solver's
    vertex blocks, the CG vectors (2 wc real columns), the triangle blocks in
    FP32 and FP64, and the mesh arrays."""
    krylov = (restart + 1) * nv * wc * 16 + (restart + 1) ** 2 * wc * 16
    vertex_blocks = 10 * nv * wc * 16
    cg = 5 * nv * 2 * wc * 8
    tri_blocks = 2 * nt * wc * 8 + 2 * nt * wc * 16
    mesh = nt * 200 + nv * 120
    return int(krylov + vertex_blocks + cg + tri_blocks + mesh)


@dataclasses.dataclass
class SolveRequest:
    """One scattering solve: far field of the sound-soft scatterer `mesh` for
    plane waves of wavenumber `kappa` from `directions` (nrhs x 3)."""
    rid: int
    coords: np.ndarray
    triangles: np.ndarray
    kappa: float
    directions: np.ndarray
    arrival: float = 0.0            # seconds after the start of the stream
    gmres_tol: float = 1e-6
    cg_tol: float = 1e-8
    mesh_key: Optional[object] = None   # requests with equal keys share a mesh

    @property
    def nrhs(self) -> int:
        return int(self.directions.shape[0])

    def footprint(self) -> int:
        return solve_footprint_bytes(self.coords.shape[0], self.triangles.shape[0], padded_rhs(self.nrhs))


@dataclasses.dataclass
class SolveResult:
    rid: int
    far_field: np.ndarray           # meas_count x nrhs complex128
    arrival: float
    start: float
    finish: float
    slot: int
    gmres_iterations: int
    gmres_relative_residual: float
    converged: bool

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


class Scheduler:
    """FIFO admission of requests to `slots` workers under a device-memory
    budget.  take() blocks until the oldest waiting request fits (a slot is free
    and the running footprints plus its own stay within the budget); a request
    larger than the whole budget is admitted alone.  Thread-safe."""

    def __init__(self, slots: int, budget_bytes: int):
        if slots < 1:
            raise ValueError("at least one slot")
        self.slots = slots
        self.budget = int(budget_bytes)
        self._pending: collections.deque = collections.deque()
        self._running: dict = {}
        self._used = 0
        self._closed = False
        self._cv = threading.Condition()
        self.peak_bytes = 0
        self.peak_running = 0

    def submit(self, req) -> None:
        with self._cv:
            self._pending.append(req)
            self._cv.notify_all()

    def close(self) -> None:
        """No more submissions: take() returns None once the queue is empty."""
        with self._cv:
            self._closed = True
            self._cv.notify_all()

    def _fits(self, req) -> bool:
        if len(self._running) >= self.slots:
            return False
        fp = req.footprint()
        return self._used + fp <= self.budget or not self._running

    def take(self, slot: int):
        with self._cv:
            while True:
                if self._pending and self._fits(self._pending[0]):
                    req = self._pending.popleft()
                    fp = req.footprint()
                    self._running[req.rid] = (slot, fp)
                    self._used += fp
                    self.peak_bytes = max(self.peak_bytes, self._used)
                    self.peak_running = max(self.peak_running, len(self._running))
                    self._cv.notify_all()
                    return req
                if self._closed and not self._pending:
                    return None
                self._cv.wait()

    def done(self, req) -> None:
        with self._cv:
            _, fp = self._running.pop(req.rid)
            self._used -= fp
            self._cv.notify_all()

    @property
    def running(self) -> int:
        with self._cv:
            return len(self._running)


def percentile(values, q: float) -> float:
    v = np.sort(np.asarray(values, dtype=np.float64))
    if v.size == 0:
        return float("nan")
    return float(np.percentile(v, q))


class SolveServer:
    """Slots of resident contexts serving SolveRequests (see module docstring).

    meas_directions: far-field directions (shared by all requests).
    slots: concurrent solves; budget_bytes: device-memory admission budget
    (default: half the free device memory at start-up).
    apply_mode: APPLY_TC (default) or APPLY_FP32; graphs: replay the solver's
    inner operators as CUDA graphs; pack (default off, tensor-core form): the
    slots' operator applies of small problems share one persistent launch
    (helmholtz.Packer, waiting at most pack_wait_us for the other solves in
    progress).  Off by default because it measured no faster: the slots' own
    streams already run small solves' kernels side by side on the GPU, and the
    packer's rendezvous of the host threads costs about what a shared launch
    saves (level-4 stream: 0.74-1.02x of the server without it, levels 4-6:
    0.97x).  autotune (default on): tune the dense
    kernel per problem shape (mesh size, right-hand-side count); the library
    caches the choice per shape for the process, so each shape is timed once.
    """

    def __init__(self, meas_directions, slots: int = 6, budget_bytes: Optional[int] = None, apply_mode=None,
                 graphs: bool = True, autotune: bool = True, device: int = 0,
                 executor: Optional[Callable] = None, pack: bool = False, pack_wait_us: int = 2000):
        from ._capi import APPLY_TC
        self.meas = np.ascontiguousarray(np.asarray(meas_directions, dtype=np.float64).reshape(-1, 3))
        self.slots = slots
        self.apply_mode = APPLY_TC if apply_mode is None else apply_mode
        self.graphs = graphs
        self.autotune = autotune
        self.device = device
        if budget_bytes is None:
            budget_bytes = self._default_budget(device)
        self.scheduler = Scheduler(slots, budget_bytes)
        self._executor = executor or self._solve_on_slot
        self._contexts: dict = {}
        self.packer = None
        if pack and self.apply_mode == APPLY_TC and executor is None:
            from .helmholtz import Packer
            self.packer = Packer(device, pack_wait_us)
        self._slot_mesh: dict = {}
        self._tuned: dict = {}          # slot -> problem shape whose tuned settings the context holds
        self.results: dict = {}
        self._lock = threading.Lock()
        self._t0 = 0.0

    @staticmethod
    def _default_budget(device: int) -> int:
        try:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            return int(free // 2)
        except Exception:
            return 64 << 30

    # ---- the GPU executor ------------------------------------------------------
    def _context(self, slot: int, req: SolveRequest):
        from .helmholtz import Helmholtz_CUDA
        H = self._contexts.get(slot)
        if H is None:
            H = Helmholtz_CUDA(req.coords, req.triangles, self.meas, device=self.device)
            H.SetApplyMode(self.apply_mode)
            H.SetGraphs(self.graphs)
            if self.packer is not None:
                H.SetPacker(self.packer)
            self._contexts[slot] = H
            self._slot_mesh[slot] = id(req) if req.mesh_key is None else req.mesh_key
            return H
        key = id(req) if req.mesh_key is None else req.mesh_key
        if self._slot_mesh.get(slot) != key:
            H.SetMesh(req.coords, req.triangles)
            self._slot_mesh[slot] = key
        return H

    def _solve_on_slot(self, slot: int, req: SolveRequest):
        from .helmholtz import WaveType
        H = self._context(slot, req)
        wcs = padded_rhs(req.nrhs)
        dirs = np.empty((wcs, 3))
        dirs[: req.nrhs] = req.directions
        dirs[req.nrhs:] = req.directions[0]          # padding columns, discarded
        kap = np.array([req.kappa], dtype=np.float64)
        shape = (req.triangles.shape[0], req.coords.shape[0], wcs)
        if self.autotune and self._tuned.get(slot) != shape:
            # the solve's operator structure (mixed BIE).  The library caches the choice per shape for the
            # process, so only a shape's first request times anything; later ones apply the cached choice
            # (a slot that served another shape in between must not keep that shape's settings).
            coeff = np.array([[0.5, -1j * req.kappa, 1.0, 0.0]])
            H.LoadBoundaryOperators_PL(kap, coeff, wcs, wcs)
            H.Autotune(self.apply_mode, repeats=1)
            H.UnloadBoundaryOperators_PL()
            self._tuned[slot] = shape
        F = np.zeros((self.meas.shape[0], wcs), complex)
        H.FarField(kap, dirs, F, WaveType.Plane, req.cg_tol, req.gmres_tol)
        st = H.LastSolveStats()
        return F[:, : req.nrhs].copy(), st

    # ---- the loop --------------------------------------------------------------
    def _worker(self, slot: int):
        while True:
            req = self.scheduler.take(slot)
            if req is None:
                return
            start = time.perf_counter() - self._t0
            try:
                F, st = self._executor(slot, req)
            finally:
                self.scheduler.done(req)
            finish = time.perf_counter() - self._t0
            res = SolveResult(req.rid, F, req.arrival, start, finish, slot, int(st["gmres_iterations"]),
                              float(st["gmres_relative_residual"]), bool(st["gmres_converged"]))
            with self._lock:
                self.results[req.rid] = res

    def run(self, requests, realtime: bool = True) -> dict:
        """Serve `requests` (arriving at their `arrival` times when `realtime`,
        else all at once) and return {rid: SolveResult}."""
        self.results = {}
        self.scheduler = Scheduler(self.slots, self.scheduler.budget)
        reqs = sorted(requests, key=lambda r: r.arrival)
        self._t0 = time.perf_counter()
        errors = []

        def guard(fn):
            def run():
                try:
                    fn()
                except BaseException as e:   # surfaced by run()
                    errors.append(e)
                    self.scheduler.close()
            return run

        workers = [threading.Thread(target=guard(lambda s=s: self._worker(s)), daemon=True)
                   for s in range(self.slots)]
        for w in workers:
            w.start()
        for r in reqs:
            if realtime:
                delay = r.arrival - (time.perf_counter() - self._t0)
                if delay > 0:
                    time.sleep(delay)
            else:
                r.arrival = time.perf_counter() - self._t0
            self.scheduler.submit(r)
        self.scheduler.close()
        for w in workers:
            w.join()
        if errors:
            raise errors[0]
        return dict(self.results)

    def pack_stats(self) -> dict:
        """Packed launches and the problems they carried (zeros without packing)."""
        return self.packer.stats() if self.packer is not None else {"launches": 0, "problems": 0}

    def close(self):
        for H in self._contexts.values():
            if self.packer is not None:
                H.SetPacker(None)
            H.close()
        self._contexts.clear()
        if self.packer is not None:
            self.packer.close()
            self.packer = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def summarize(results: dict) -> dict:
    """Throughput and latency of a served stream."""
    rs = list(results.values())
    if not rs:
        return {}
    lat = [r.latency for r in rs]
    span = max(r.finish for r in rs) - min(r.arrival for r in rs)
    return {"requests": len(rs), "solves_per_s": len(rs) / span if span > 0 else float("nan"),
            "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)), "makespan_s": span,
            "converged": int(sum(r.converged for r in rs))}


def make_stream(n: int, rate: float, levels=(4, 5, 6), kappa_range=(1.0, 10.0), rhs_range=(1, 64),
                degree: int = 8, amplitude: float = 0.1, seed: int = 0):
    """Synthetic request stream: Poisson arrivals at `rate` per second; each
    mesh an icosphere of a level drawn uniformly from `levels`, radially
    perturbed by 1 + amplitude * S / max|S| (S a random real spherical-harmonic
    sum of degree <= `degree`); kappa uniform in `kappa_range`; a uniform
    number of plane-wave directions in `rhs_range`, random unit vectors."""
    from .meshes import sh_perturbed_sphere
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        level = int(rng.choice(levels))
        coords, tris = sh_perturbed_sphere(level, degree, amplitude, seed=seed * 100003 + rid)
        k = float(rng.uniform(*kappa_range))
        nrhs = int(rng.integers(rhs_range[0], rhs_range[1] + 1))
        d = rng.standard_normal((nrhs, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        out.append(SolveRequest(rid, coords, tris, k, d, arrival=t))
    return out
