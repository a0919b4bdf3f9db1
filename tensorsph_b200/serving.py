"""Serving simulations from a request stream with continuous batching.

Requests arrive as a Poisson stream (seeded); each names a case type, a
particle count and a simulated time.  A ``Server`` owns one ``BatchEngine``
whose arena is the HBM budget: a request is admitted as soon as it has
arrived and its footprint (fluid rows, wall rows, cells, a case slot) fits in
what the running cases leave free -- first fit in arrival order, so a small
request can pass a large one that is still waiting.  Admitted cases stay on
the device, run together (one CUDA graph step for all), and retire the
moment they reach their own step count, which frees room for the next ones.

The engine advances in chunks of at most ``max_chunk`` steps that never pass
the next completion, so a case runs exactly its own number of steps and each
result equals the same request run alone (bitwise: see the engine).  The host
enqueues chunks, retirements and admissions on the engine stream without
waiting in between (one chunk in flight ahead of the one being prepared), and
the engine absorbs a change of the batch by updating its instantiated step
graph in place.  Latency is from arrival to the device time at which the
request's last step completed; ``run_serial`` serves the same stream one
request at a time in arrival order with the single-case engine.

Case types: ``dam_break_2d`` (1 : 2 column in a 4 x 1.5 tank, dam_break.py),
``column_3d`` (hydrostatic 3-D column filling a square tank,
dam_break_3d.py), both with c0 = 10 sqrt(2 g H) and acoustic CFL 0.25, and
``shear_3d`` (triply periodic shear decay u_x = 1e-3 sin(2 pi z) in a unit
cube, nu = 1e-2, c0 = 1); each sized by its particle count.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import math
import time

import numpy as np

from .engine import MAX_ROWS, BatchEngine, CaseSpec, dam_break_2d_case, dam_break_3d_case, engine_bytes

__all__ = ["Request", "request_stream", "request_spec", "Server", "capacities_for_budget",
           "run_serial", "percentiles"]

CASE_TYPES = ("dam_break_2d", "column_3d", "shear_3d")


@dataclass
class Request:
    rid: int
    arrival: float          # s after the stream starts
    kind: str
    particles: int          # requested fluid particle count
    sim_time: float         # requested simulated time (s)
    height: float = 1.0     # column height (m)
    spec: CaseSpec | None = field(default=None, repr=False)
    steps: int = 0
    admitted: float = -1.0
    finished: float = -1.0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_stream(n: int, *, rate: float = 20.0, seed: int = 0, n_min: float = 1e3,
                   n_max: float = 2e6, t_min: float = 0.1, t_max: float = 1.0,
                   time_scale: float = 1.0, kinds=CASE_TYPES) -> list[Request]:
    """``n`` requests: Poisson arrivals at ``rate``/s, type uniform over
    ``kinds``, particle count log-uniform in [n_min, n_max], simulated time
    uniform in [t_min, t_max] times ``time_scale`` (a scale < 1 keeps a
    benchmark short), column height uniform in [0.5, 2] m."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        kind = kinds[int(rng.integers(len(kinds)))]
        parts = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        sim = float(rng.uniform(t_min, t_max)) * time_scale
        height = float(rng.uniform(0.5, 2.0))
        out.append(Request(i, t, kind, parts, sim, height))
    return out


def request_spec(req: Request) -> CaseSpec:
    """The case of a request, sized to its particle count."""
    g = 9.81
    c0 = 10.0 * math.sqrt(2.0 * g * req.height)
    if req.kind == "dam_break_2d":
        from .dam_break import DamBreakConfig
        w = 0.5 * req.height
        dx = math.sqrt(w * req.height / req.particles)
        h = 1.3 * dx
        cfg = DamBreakConfig(dx=dx, column_width=w, column_height=req.height, pool_width=4.0 * w,
                             tank_height=1.5 * req.height, sound_speed=c0, viscosity=1e-6,
                             dt=0.25 * h / c0, max_courant=0.25)
        spec = dam_break_2d_case(cfg, label=f"r{req.rid}:{req.kind}")
    elif req.kind == "column_3d":
        from .dam_break_3d import DamBreak3DConfig
        w = 0.5 * req.height
        dx = (w * w * req.height / req.particles) ** (1.0 / 3.0)
        h = 1.3 * dx
        cfg = DamBreak3DConfig(dx=dx, pool_width=w, tank_depth=w, tank_height=1.2 * req.height,
                               column_width=w, column_depth=w, column_height=req.height,
                               sound_speed=c0, viscosity=1e-6, dt=0.25 * h / c0,
                               max_courant=0.25)
        spec = dam_break_3d_case(cfg, label=f"r{req.rid}:{req.kind}")
    elif req.kind == "shear_3d":
        from .engine import shear_decay_case
        n = max(8, int(round(req.particles ** (1.0 / 3.0))))
        spec = shear_decay_case(n, seed=req.rid, label=f"r{req.rid}:{req.kind}")
    else:
        raise ValueError(f"unknown case type {req.kind!r}")
    req.spec = spec
    req.steps = max(1, int(round(req.sim_time / spec.dt)))
    return spec


def percentiles(values, qs=(50, 99)) -> dict:
    if not values:
        return {f"p{q}": None for q in qs}
    return {f"p{q}": float(np.percentile(np.asarray(values), q)) for q in qs}


def capacities_for_budget(budget_bytes: float, *, max_cases: int = 64,
                          max_neighbors: int = 160) -> dict:
    """Engine capacities whose arena fits ``budget_bytes``: fluid rows with one
    wall row per two fluid rows and two cells per fluid row (the mix of the
    case types served here)."""
    probe = dict(max_cells=1, max_cases=max_cases, max_neighbors=max_neighbors, diag_ring=4,
                 max_obstacle=0)
    base = engine_bytes(max_fluid=1, max_wall=1, **probe)
    m = 1 << 20
    per_f = (engine_bytes(max_fluid=m, max_wall=1, **probe) - base) / m
    per_w = (engine_bytes(max_fluid=1, max_wall=m, **probe) - base) / m
    per_c = (engine_bytes(max_fluid=1, max_wall=1, **dict(probe, max_cells=m)) - base) / m
    room = max(float(budget_bytes) - base, 0.0)
    max_fluid = int(room / (per_f + per_w / 2.0 + 2.0 * per_c))
    max_fluid = min(max_fluid, (MAX_ROWS * 2) // 3)   # fluid + wall rows <= MAX_ROWS
    return dict(max_fluid=max_fluid, max_wall=max(max_fluid // 2, 1), max_cells=2 * max_fluid,
                max_cases=max_cases, max_neighbors=max_neighbors, diag_ring=4, max_obstacle=0)


class Server:
    """Continuous-batching server over one fixed-budget engine."""

    def __init__(self, *, budget_bytes: float, max_cases: int = 64, max_neighbors: int = 160,
                 device=None):
        self.capacity = capacities_for_budget(budget_bytes, max_cases=max_cases,
                                              max_neighbors=max_neighbors)
        self.engine = BatchEngine(**self.capacity, device=device)
        self.budget_bytes = float(budget_bytes)
        self.engine_bytes = self.engine.nbytes

    def close(self):
        self.engine.close()

    def serve(self, requests, *, max_chunk: int = 64, keep_results: bool = False) -> dict:
        """Serve the stream in real time; returns per-request latencies and
        aggregate throughput.

        The host never waits for the device between chunks: a chunk's steps,
        the retirement of the cases it completes and the admission of the
        requests that have arrived are all enqueued on the engine stream, and
        the host only waits for the chunk before the one in flight, so the
        device always has the next chunk queued.  A request's completion time
        is the device time (CUDA events on the engine stream, from an event
        recorded when serving starts) of the end of its last chunk."""
        import torch
        eng = self.engine
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            if r.spec is None:
                request_spec(r)
        waiting: list[Request] = []
        active: dict[int, tuple[Request, int]] = {}   # case id -> (request, steps left)
        results = {}
        updates = 0
        steps_run = 0
        blocked = set()      # requests that arrived and had to wait for room
        stats0 = eng.graph_stats()
        inflight: list = []  # (event, [(request, last meter row, state or None)])
        t0 = time.perf_counter()
        start = torch.cuda.Event(enable_timing=True)
        start.record(eng.stream)

        def retire(entry):
            ev, done = entry
            ev.synchronize()
            at = start.elapsed_time(ev) / 1e3
            for r, row, state in done:
                if float(row[0, 13]) != 0.0:
                    raise FloatingPointError(f"request {r.rid} went non-finite")
                r.finished = at
                if state is not None:
                    results[r.rid] = [t.cpu() for t in state]

        i = 0
        while i < len(pending) or waiting or active or inflight:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival <= now:
                waiting.append(pending[i])
                i += 1
            for r in list(waiting):
                if eng.fits(r.spec):
                    cid = eng.add(r.spec)
                    r.admitted = time.perf_counter() - t0
                    active[cid] = (r, r.steps)
                    waiting.remove(r)
                else:
                    blocked.add(r.rid)
            if not active:
                while inflight:
                    retire(inflight.pop(0))
                if waiting and i >= len(pending):
                    raise RuntimeError(f"request {waiting[0].rid} can never fit the budget")
                if i < len(pending):
                    time.sleep(max(0.0, pending[i].arrival - (time.perf_counter() - t0)))
                continue
            chunk = min(max_chunk, min(left for _, left in active.values()))
            eng.step(chunk)
            steps_run += chunk
            updates += chunk * sum(r.spec.n_fluid for r, _ in active.values())
            done = []
            for cid in list(active):
                r, left = active[cid]
                left -= chunk
                if left == 0:
                    row = eng.diagnostics(cid, eng.steps_of[cid] - 1, 1)
                    state = eng.read(cid) if keep_results else None
                    eng.remove(cid)
                    done.append((r, row, state))
                    del active[cid]
                else:
                    active[cid] = (r, left)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(eng.stream)
            inflight.append((ev, done))
            while len(inflight) > 1:
                retire(inflight.pop(0))
        while inflight:
            retire(inflight.pop(0))
        end = torch.cuda.Event(enable_timing=True)
        end.record(eng.stream)
        end.synchronize()
        wall = max(time.perf_counter() - t0, start.elapsed_time(end) / 1e3)
        lat = [r.latency for r in pending]
        stats = eng.graph_stats()
        return {"requests": len(pending), "wall_s": wall, "updates": updates,
                "updates_per_s": updates / wall, "engine_steps": steps_run,
                "latency_s": percentiles(lat), "results": results,
                "admissions_blocked": len(blocked),
                "graph_instantiations": stats["instantiations"] - stats0["instantiations"],
                "graph_updates": stats["updates"] - stats0["updates"]}


def run_serial(requests, *, max_neighbors: int = 160, device=None, keep_results: bool = False) -> dict:
    """The same stream served one request at a time, in arrival order, each in
    a single-case engine sized to it (the plain drop-in)."""
    from .engine import capacity_for
    pending = sorted(requests, key=lambda r: r.arrival)
    for r in pending:
        if r.spec is None:
            request_spec(r)
    results = {}
    updates = 0
    t0 = time.perf_counter()
    lat = []
    for r in pending:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        eng = BatchEngine(**capacity_for([r.spec], max_neighbors=max_neighbors, diag_ring=4),
                          device=device)
        cid = eng.add(r.spec)
        eng.step(r.steps)
        eng.stream.synchronize()
        if keep_results:
            results[r.rid] = [t.cpu() for t in eng.read(cid)]
        eng.close()
        updates += r.steps * r.spec.n_fluid
        lat.append(time.perf_counter() - t0 - r.arrival)
    wall = time.perf_counter() - t0
    return {"requests": len(pending), "wall_s": wall, "updates": updates,
            "updates_per_s": updates / wall, "latency_s": percentiles(lat), "results": results}
