"""Batched and served forms: many independent water boxes advanced at once
on one GPU.

Every admitted request owns a GpuSystem (its own CUDA stream, resident
coordinates, velocities, neighbour list and PME grids).  A request is either
one energy + force evaluation or an MD segment (LangevinLeapfrog by default).
Admission is continuous: a request is started as soon as a slot is free and
its footprint estimate fits in the device-memory budget, while the segments
already admitted keep running; their kernels overlap on the device because
each system runs on its own stream and the library releases the GIL inside
every blocking call.  The plain form is the same loop with one slot.

Each result is a pure function of the request (fixed-point force sums and a
counter-based Langevin noise), so it is bit-identical alone and in the mix.
"""
from __future__ import annotations

import dataclasses
import math
import queue
import threading
import time

import numpy as np

from . import systems
from .engine import (Context, ForceFactory, GpuSystem, LangevinLeapfrogIntegrator,
                     SystemEnsemble,
                     LeapfrogIntegrator, footprint_estimate)

WATER_DENSITY = 0.0334  # waters per A^3
RC, ALPHA, ORDER, LJ_SWITCHON, SPACING, SKIN = 9.0, 0.35, 4, 8.0, 1.0, 1.3


def fft_size(n: int) -> int:
    """Smallest 2^a 3^b 5^c >= n."""
    m = max(1, n)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


@dataclasses.dataclass
class Request:
    """One unit of served work on a seeded TIP3P box."""
    rid: int
    n_waters: int
    seed: int
    kind: str = "segment"        # "segment" | "evaluate"
    steps: int = 1000
    integrator: str = "langevin"  # "langevin" | "leapfrog"
    timestep: float = 1.0
    temperature: float = 300.0
    gamma: float = 5.0
    arrival: float = 0.0          # seconds after the stream starts
    system: systems.MolecularSystem | None = None  # the client's input
    # filled in by the server
    t_start: float = 0.0
    t_done: float = 0.0
    energies: np.ndarray | None = None
    positions: np.ndarray | None = None
    forces: np.ndarray | None = None
    error: str | None = None

    @property
    def n_atoms(self) -> int:
        return 3 * self.n_waters

    @property
    def edge(self) -> float:
        return (self.n_waters / WATER_DENSITY) ** (1.0 / 3.0)

    @property
    def grid(self) -> int:
        return fft_size(int(math.ceil(self.edge / SPACING)))

    def footprint(self) -> int:
        L = self.edge
        g = self.grid
        return footprint_estimate(self.n_atoms, (L, L, L), RC + SKIN, (g, g, g))

    def latency(self) -> float:
        return self.t_done - self.arrival

    def prepare(self) -> "Request":
        """Builds the request's input system (the client's side of a
        request: the server receives a ready topology and coordinates)."""
        if self.system is None:
            self.system = systems.water_box_for_density(self.n_waters, WATER_DENSITY, self.seed,
                                                        jitter=0.2)
        return self


def force_lines(grid: int) -> list[str]:
    return ["Bond", "Angle",
            f"LennardJones -algorithm NonbondedCutoff -switchingFunction C2 "
            f"-switchon {LJ_SWITCHON} -cutoff {RC} -cutoff {RC}",
            f"Coulomb -algorithm PMEwald -alpha {ALPHA} -cutoff {RC} -order {ORDER} "
            f"-gridsize {grid} {grid} {grid}"]


def build(ctx: Context, req: Request, precision: str = "mixed") -> GpuSystem:
    gs = GpuSystem(ctx, req.prepare().system, precision)
    ff = ForceFactory(gs, RC)
    for line in force_lines(req.grid):
        ff.make(line)
    return gs


class ShellPool:
    """Idle systems kept for reuse.  Requests on boxes of the same shape
    (water count, hence edge, grid and topology) share a key; a request
    whose key has an idle shell takes it instead of creating a system: its
    positions, velocities and Langevin step counter are set, and the
    shell's device buffers, pair list, cuFFT plans and captured step graphs
    are reused.  A request's results are the same in a reused shell as in
    a new system (every list is built afresh from the new positions).
    Idle shells beyond cap_bytes (by their footprint estimates) are closed,
    the least recently used first."""

    def __init__(self, ctx: Context, cap_bytes: int):
        self.ctx = ctx
        self.cap = int(cap_bytes)
        self.lock = threading.Lock()
        self.idle: dict = {}  # key -> [GpuSystem]
        self.lru: list = []   # (key, footprint) of idle shells, oldest first
        self.held = 0
        self.reused = 0
        self.created = 0

    @staticmethod
    def key(req: Request):
        return (req.n_waters, req.grid)

    def acquire(self, req: Request) -> GpuSystem:
        k = self.key(req)
        gs = None
        with self.lock:
            if self.idle.get(k):
                gs = self.idle[k].pop()
                for q, (kk, fp) in enumerate(self.lru):
                    if kk == k:
                        self.held -= fp
                        del self.lru[q]
                        break
                self.reused += 1
            else:
                self.created += 1
        if gs is None:
            return build(self.ctx, req)
        sysm = req.prepare().system
        gs.set_positions(sysm.pos)
        gs.set_velocities(sysm.vel)
        gs.set_step(0)
        return gs

    def release(self, req: Request, gs: GpuSystem) -> None:
        k = self.key(req)
        fp = req.footprint()
        evict = []
        with self.lock:
            if fp > self.cap:
                evict.append(gs)
            else:
                self.idle.setdefault(k, []).append(gs)
                self.lru.append((k, fp))
                self.held += fp
                while self.held > self.cap and self.lru:
                    kk, f = self.lru.pop(0)
                    evict.append(self.idle[kk].pop(0))
                    self.held -= f
        for g in evict:
            g.close()

    def close(self) -> None:
        with self.lock:
            shells = [g for v in self.idle.values() for g in v]
            self.idle.clear()
            self.lru.clear()
            self.held = 0
        for g in shells:
            g.close()


def execute(ctx: Context, req: Request, keep_positions: bool = True,
            pool: ShellPool | None = None) -> Request:
    """Runs one request to completion on the calling thread (in a shell
    from `pool` when one is given)."""
    gs = pool.acquire(req) if pool is not None else build(ctx, req)
    ok = False
    try:
        if req.kind == "evaluate":
            e, _ = gs.evaluate()
            req.energies = e
            req.forces = gs.forces_total()
        else:
            if req.integrator == "langevin":
                integ = LangevinLeapfrogIntegrator(req.timestep, req.temperature, req.gamma,
                                                   seed=req.seed)
            else:
                integ = LeapfrogIntegrator(req.timestep)
            integ.run(gs, req.steps)
            req.energies = gs.energies()[0]
            if keep_positions:
                req.positions = gs.positions()
        ok = True
    finally:
        if pool is not None and ok:
            pool.release(req, gs)
        else:
            gs.close()
    return req


class Server:
    """Continuous-batching request loop over one device.

    slots: requests in flight at once (one worker thread each);
    mem_fraction: share of the device memory free at start-up that admitted
    requests may hold (by their footprint estimates);
    pool_fraction: share of it kept for idle shells (ShellPool; 0: every
    request creates and frees its own system)."""

    def __init__(self, ctx: Context, slots: int = 16, mem_fraction: float = 0.8,
                 pool_fraction: float = 0.2):
        self.ctx = ctx
        self.slots = slots
        free, _ = ctx.mem_info()
        total = int(free * mem_fraction)
        self.pool = ShellPool(ctx, int(total * pool_fraction)) if pool_fraction > 0 else None
        self.budget = total - (self.pool.cap if self.pool else 0)
        self.in_use = 0
        self.lock = threading.Condition()
        self.admit_q: queue.Queue = queue.Queue()
        self.done: list[Request] = []
        self.peak_in_flight = 0
        self.in_flight = 0
        self.peak_in_use = 0

    def _worker(self):
        while True:
            req = self.admit_q.get()
            if req is None:
                return
            try:
                execute(self.ctx, req, pool=self.pool)
            except Exception as ex:  # reported per request, the loop goes on
                req.error = str(ex)[:300]
            req.t_done = time.perf_counter() - self.t0
            with self.lock:
                self.in_use -= req._fp
                self.in_flight -= 1
                self.done.append(req)
                self.lock.notify_all()

    def run(self, requests: list[Request], realtime: bool = True) -> dict:
        """Serves the requests (in arrival order; with realtime the arrival
        times are honoured) and returns throughput and latency figures."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            r.prepare()  # inputs arrive ready-made; building them is not timed
            r._fp = r.footprint()
            if r._fp > self.budget:
                raise ValueError(f"request {r.rid} needs {r._fp} B, over the budget {self.budget}")
        workers = [threading.Thread(target=self._worker, daemon=True) for _ in range(self.slots)]
        for w in workers:
            w.start()
        self.t0 = time.perf_counter()
        for r in reqs:
            if realtime:
                wait = r.arrival - (time.perf_counter() - self.t0)
                if wait > 0:
                    time.sleep(wait)
            with self.lock:
                # admit when a slot and the memory are free
                while self.in_flight >= self.slots or self.in_use + r._fp > self.budget:
                    self.lock.wait()
                self.in_use += r._fp
                self.in_flight += 1
                self.peak_in_flight = max(self.peak_in_flight, self.in_flight)
                self.peak_in_use = max(self.peak_in_use, self.in_use)
            r.t_start = time.perf_counter() - self.t0
            self.admit_q.put(r)
        with self.lock:
            while len(self.done) < len(reqs):
                self.lock.wait()
        wall = time.perf_counter() - self.t0
        for _ in workers:
            self.admit_q.put(None)
        for w in workers:
            w.join()
        out = summarize(reqs, wall, self.slots, self.peak_in_flight)
        out["peak_footprint_bytes"] = self.peak_in_use
        out["budget_bytes"] = self.budget
        if self.pool is not None:
            out["shells_reused"] = self.pool.reused
            out["shells_created"] = self.pool.created
        return out

    def close(self) -> None:
        if self.pool is not None:
            self.pool.close()


class Ensemble:
    """Many resident boxes advanced together, in three forms:

    - "batched": one engine.SystemEnsemble; every kernel of a step is one
      launch over all members (pair-kernel splits per size bucket from the
      autotuner), each segment one captured CUDA graph;
    - "streams": each member's own pmgpu_run segment enqueued on its own
      stream before any is waited for, so the members' kernels overlap;
    - "plain": the members one at a time.

    Every member keeps its state on the device between segments."""

    def __init__(self, ctx: Context, requests: list[Request], tuner=None):
        self.requests = requests
        self.members = [build(ctx, r.prepare()) for r in requests]
        self.integ = [LeapfrogIntegrator(r.timestep) if r.integrator == "leapfrog" else
                      LangevinLeapfrogIntegrator(r.timestep, r.temperature, r.gamma, seed=r.seed)
                      for r in requests]
        self.batch = None
        self.splits = None
        self.tuner = tuner

    def _batched(self) -> SystemEnsemble:
        if self.batch is None:
            p0 = self.integ[0].p
            for it in self.integ:
                if (it.p.kind, it.p.timestep_fs, it.p.temperature, it.p.gamma_ps,
                        it.p.seed) != (p0.kind, p0.timestep_fs, p0.temperature, p0.gamma_ps,
                                       p0.seed):
                    raise ValueError("the batched form runs one integrator for all members")
            self.batch = SystemEnsemble(self.members)
            if self.tuner is not None:
                self.splits = self.tuner.apply(self.batch)
        return self.batch

    def run(self, steps: int, mode: str = "batched") -> float:
        """One segment of `steps` MD steps for every member; wall seconds."""
        if mode == "batched":
            ens = self._batched()
            t0 = time.perf_counter()
            ens.run(self.integ[0], steps)
            return time.perf_counter() - t0
        t0 = time.perf_counter()
        if mode == "plain":
            for gs, it in zip(self.members, self.integ):
                it.run(gs, steps)
        elif mode == "streams":
            for gs, it in zip(self.members, self.integ):
                it.run_async(gs, steps)
            for gs, it in zip(self.members, self.integ):
                it.wait(gs)
        else:
            raise ValueError(f"unknown ensemble form {mode!r}")
        return time.perf_counter() - t0

    def info(self) -> dict | None:
        return self.batch.info() if self.batch is not None else None

    def energies(self) -> list[np.ndarray]:
        return [gs.energies()[0] for gs in self.members]

    def positions(self) -> list[np.ndarray]:
        return [gs.positions() for gs in self.members]

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        for gs in self.members:
            gs.close()
        self.members = []

    @property
    def atoms(self) -> int:
        return sum(r.n_atoms for r in self.requests)


def summarize(reqs: list[Request], wall: float, slots: int, peak: int) -> dict:
    ok = [r for r in reqs if r.error is None]
    lat = np.array([r.latency() for r in ok]) if ok else np.zeros(1)
    md_ns = sum(r.steps * r.timestep * 1e-6 for r in ok if r.kind == "segment")
    atom_steps = sum(r.n_atoms * (r.steps if r.kind == "segment" else 1) for r in ok)
    return {
        "requests": len(reqs), "failed": len(reqs) - len(ok), "slots": slots,
        "peak_in_flight": peak, "wall_s": wall,
        "ns_per_day": md_ns * 86400.0 / wall,
        "atom_steps_per_s": atom_steps / wall,
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
    }


def request_stream(n: int, seed: int, min_atoms: int = 500, max_atoms: int = 50000,
                   eval_fraction: float = 0.3, steps: int = 1000,
                   rate_per_s: float | None = None) -> list[Request]:
    """A seeded request stream: atom counts log-uniform in [min, max]
    (rounded to whole waters), a share of single evaluations, the rest MD
    segments; Poisson arrivals at rate_per_s (None: all at time 0)."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for k in range(n):
        atoms = math.exp(rng.uniform(math.log(min_atoms), math.log(max_atoms)))
        nw = max(1, int(round(atoms / 3)))
        kind = "evaluate" if rng.uniform() < eval_fraction else "segment"
        if rate_per_s:
            t += rng.exponential(1.0 / rate_per_s)
        out.append(Request(rid=k, n_waters=nw, seed=int(rng.integers(1 << 31)), kind=kind,
                           steps=steps if kind == "segment" else 0, arrival=t))
    return out


def ensemble(n_boxes: int, seed: int, min_waters: int = 100, max_waters: int = 1000,
             steps: int = 50) -> list[Request]:
    """The batched ensemble: boxes with water counts log-uniform in
    [min_waters, max_waters], one MD segment each, all available at once."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_boxes):
        nw = int(round(math.exp(rng.uniform(math.log(min_waters), math.log(max_waters)))))
        out.append(Request(rid=k, n_waters=nw, seed=int(rng.integers(1 << 31)), steps=steps,
                           integrator="leapfrog"))
    return out
