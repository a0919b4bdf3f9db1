"""Batched ensemble of independent 2-D droplet-impact cases on one GPU.

An ensemble draws its cases from one seed: drop radius R ~ U[0.02, 0.08] m at
dx = R / 20, pool depth ~ U[2R, 6R], pool width 8R and impact speed
U ~ U[1, 5] m/s (rho0 = 1000).  Every case gets c0 = 10 max(U, sqrt(2 g d))
(Mach <= 0.1) and dt at acoustic CFL 0.25; the rest is the reference
``Config`` (droplet_impact.py:55-269) with CSF surface tension sigma =
0.0728 N/m (consistent scheme, quadratic curvature fit).  With dx tied to R
the particle count depends on the depth ratio only: 7.7k (pool 2R) to 20.5k
(pool 6R) fluid.

``run_batched`` advances all cases in one engine (one CUDA graph per step for
the whole ensemble); ``run_plain`` runs the same cases one at a time, each in
an engine of its own -- the single-case path -- and the two report
fluid particle-updates/s.  ``autotune`` picks the pair-kernel block size and
the Verlet skin (which sets the cell size) by timing a sample of the cases.
"""
from __future__ import annotations

from dataclasses import dataclass, replace
import math
import time

import numpy as np
import torch

from .droplet_impact import Config
from .engine import BatchEngine, CaseSpec, capacity_for, droplet_impact_case

__all__ = ["DropletDraw", "draw_ensemble", "droplet_config", "ensemble_specs", "autotune",
           "run_batched", "run_plain"]


@dataclass(frozen=True)
class DropletDraw:
    radius: float
    depth: float
    speed: float


def draw_ensemble(n: int = 256, seed: int = 0) -> list[DropletDraw]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        r = float(rng.uniform(0.02, 0.08))
        d = float(rng.uniform(2.0 * r, 6.0 * r))
        u = float(rng.uniform(1.0, 5.0))
        out.append(DropletDraw(r, d, u))
    return out


def droplet_config(draw: DropletDraw, *, skin_factor: float = 0.25, courant: float = 0.25,
                   viscosity: float = 1.0e-6, surface_tension: float = 0.0728) -> Config:
    dx = draw.radius / 20.0
    c0 = 10.0 * max(draw.speed, math.sqrt(2.0 * 9.81 * draw.depth))
    h = 1.3 * dx
    return Config(dx=dx, pool_width=8.0 * draw.radius, pool_depth=draw.depth,
                  drop_radius=draw.radius, drop_center_y=draw.depth + draw.radius + 1.5 * dx,
                  sound_speed=c0, viscosity=viscosity, dt=courant * h / c0, max_courant=courant,
                  pair_skin_factor=skin_factor, surface_tension_coefficient=surface_tension)


def ensemble_specs(draws, *, skin_factor: float = 0.25, surface_tension: float = 0.0728) -> list[CaseSpec]:
    return [droplet_impact_case(droplet_config(d, skin_factor=skin_factor,
                                               surface_tension=surface_tension),
                                drop_speed=d.speed, label=f"droplet R={d.radius:.4f}") for d in draws]


def _timed_steps(eng: BatchEngine, steps: int) -> float:
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(eng.stream)
    eng.step(steps)
    stop.record(eng.stream)
    stop.synchronize()
    return start.elapsed_time(stop) / 1e3


def run_batched(specs, steps: int, *, warmup: int = 3, block: int = 128, batch: int = 4,
                max_neighbors: int = 64, device=None) -> dict:
    """All cases in one engine; device time of ``steps`` steps after ``warmup``."""
    eng = BatchEngine(**capacity_for(specs, max_neighbors=max_neighbors, diag_ring=8), device=device)
    eng.set_block(block)
    eng.set_batch(batch)
    ids = [eng.add(s) for s in specs]
    eng.step(warmup)
    t = _timed_steps(eng, steps)
    kernels, rebuild_kernels = eng.graph_kernels()
    bad = [i for i in ids if eng.status(i)["status"]]
    nf = sum(s.n_fluid for s in specs)
    eng.close()
    return {"cases": len(specs), "fluid": nf, "steps": steps, "seconds": t,
            "updates_per_s": nf * steps / t, "kernels_per_step": kernels,
            "kernels_per_rebuild_pass": rebuild_kernels, "failed_cases": bad}


def run_plain(specs, steps: int, *, warmup: int = 3, block: int = 128, batch: int = 4,
              max_neighbors: int = 64, device=None) -> dict:
    """The same cases one at a time, each in its own single-case engine (the
    plain drop-in loop); device time summed over the cases."""
    total_t, total_u = 0.0, 0
    for s in specs:
        eng = BatchEngine(**capacity_for([s], max_neighbors=max_neighbors, diag_ring=8), device=device)
        eng.set_block(block)
        eng.set_batch(batch)
        eng.add(s)
        eng.step(warmup)
        total_t += _timed_steps(eng, steps)
        total_u += s.n_fluid * steps
        eng.close()
    return {"cases": len(specs), "fluid": sum(s.n_fluid for s in specs), "steps": steps,
            "seconds": total_t, "updates_per_s": total_u / total_t}


def autotune(draws, *, blocks=(64, 128, 256), batches=(4, 8, 16), skins=(0.15, 0.25, 0.4),
             steps: int = 30, warmup: int = 10, device=None, cache: bool = True) -> dict:
    """Time each (block, batch depth, skin) on the sample ``draws`` and return
    the fastest.

    The skin sets both the cell edge (2h + skin) and how often lists are
    rebuilt, so it is timed over enough steps to include rebuilds.  With
    ``cache`` a previous result for the same sample size and GPU
    (``tensorsph_b200.tuning``) is returned without timing, and a new one kept."""
    from . import tuning
    key = None
    if cache:
        dev = device or torch.device("cuda", torch.cuda.current_device())
        n = sum(s.n_fluid for s in ensemble_specs(draws, skin_factor=skins[0]))
        key = tuning.tuning_key(f"droplet_ensemble{len(draws)}", dim=2, particles=n, h_over_dx=1.3,
                                candidates={"skins": skins, "blocks": blocks, "batches": batches},
                                gpu=torch.cuda.get_device_name(dev))
        hit = tuning.lookup(key)
        if hit is not None:
            return {"best": hit, "trials": [], "cached": True}
    trials = []
    for skin in skins:
        specs = ensemble_specs(draws, skin_factor=skin)
        for block in blocks:
            for batch in batches:
                r = run_batched(specs, steps, warmup=warmup, block=block, batch=batch, device=device)
                trials.append({"block": block, "batch": batch, "skin_factor": skin,
                               "updates_per_s": r["updates_per_s"]})
    best = max(trials, key=lambda t: t["updates_per_s"])
    if key is not None:
        tuning.store(key, best)
    return {"best": best, "trials": trials, "cached": False}


def main(argv=None) -> None:
    """``python -m tensorsph_b200.ensemble --cases N --steps K``: run one
    batched droplet ensemble and print its device throughput."""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--skin", type=float, default=0.15)
    ap.add_argument("--block", type=int, default=64)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--sigma", type=float, default=0.0728)
    ap.add_argument("--eager", action="store_true", help="launch kernel by kernel (no graph)")
    args = ap.parse_args(argv)
    specs = ensemble_specs(draw_ensemble(args.cases, seed=args.seed), skin_factor=args.skin,
                           surface_tension=args.sigma)
    eng = BatchEngine(**capacity_for(specs, max_neighbors=64, diag_ring=8))
    eng.set_block(args.block)
    eng.set_batch(args.batch)
    for s in specs:
        eng.add(s)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(eng.stream)
    eng.step(args.steps, graph=not args.eager)
    stop.record(eng.stream)
    stop.synchronize()
    ms = start.elapsed_time(stop) / max(args.steps, 1)
    nf = sum(s.n_fluid for s in specs)
    print(f"cases {len(specs)} fluid {nf} ms/step {ms:.3f} updates/s {nf / ms * 1e3:.3e}")
    eng.close()


if __name__ == "__main__":
    main()
