"""Benchmark: fluid particle-updates/s of the 3-D dam break with a box obstacle.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Workload (one case per GPU; with N > 1 every rank runs its own replica, weak
scaling, no collective on the data path): fluid block 1.2 x 1.0 x 0.55 m at
dx = 0.0069 m (1,968,048 fluid particles) in a 3.2 x 1.0 x 1.0 m tank with
three wall layers and a 0.16 x 0.16 x 0.4 m obstacle (776k wall particles),
h = 1.3 dx, Tait rho0 = 1000, gamma = 7, c0 = 10 sqrt(2 g 0.55), Molteni
diffusion delta = 0.1, Lind shifting every step, CFL 0.25; FP32 pair
arithmetic with FP64 positions, velocities and meters.

A bench step is ``--chunk`` solver steps (default: enough that the K timed
bench steps cover at least 200 solver steps, so that the timed region holds
the neighbour-list rebuilds at their natural rate, about one per list pass
every 20-40 steps).  A solver step is one graph-launched engine step: per-case
skin test and device-side rebuild (conditional), density, diffusion + EOS,
Adami walls, force, obstacle force, Euler + clamps, shifting.

One JSON line on rank 0.  ``value`` is device-timed (CUDA events on the
engine stream, max over ranks); ``e2e`` is the same metric through the public
API from pinned host memory: engine creation from the host lattice (H2D), the
K bench steps with one device->host read of a meter row per bench step, and
the final state back to the host.  ``--impl reference`` times the reference's
own CPU code (``baseline/_ref``, torch on every host core) on a 4x coarser
rung of the same case.
"""
from __future__ import annotations

import argparse
import json
import math
import os
from pathlib import Path
import statistics
import subprocess
import sys
import time

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ALGO_BYTES_FORCE = 52      # per fluid particle: pos+mass 16, vel+rho 16, p/rho^2 4 in; acc 16 out
ALGO_BYTES_STEP = 244      # per fluid update, compulsory bytes of the whole step (3-D plain path)
ALGO_BYTES_WALL = 48       # per wall particle and step
# FP32 operations per listed neighbour of each pair pass, counted from the
# kernel source (an FMA counts 2, every other arithmetic instruction 1,
# including rsqrt, reciprocals and the integer-to-FP32 conversion of the
# fixed-point separation; a packed FP32x2 instruction counts once per
# neighbour it serves).
PAIR_FLOPS = {"density": 27, "diffusion": 50, "walls": 32, "force": 65, "concentration": 27,
              "gradient": 51}
# DRAM bytes of one force launch per fluid particle: ncu capture of the force
# pass on the dx = 0.0138 rung (241,488 fluid) at skin 0.15 h and depth 8,
# dram__bytes_read.sum + dram__bytes_write.sum divided by the fluid rows.
FORCE_TRAFFIC_PER_FLUID = 373.0
FORCE_TRAFFIC_RUNG = "dx=0.0138 (241,488 fluid), skin 0.15 h, depth 8, ncu capture scaled by fluid rows"
# What the same ncu capture shows limits the force pass (neither roof binds).
FORCE_LIMITER = ("l1: l1tex throughput 90 % of peak, data pipe 74 % of elapsed cycles, long-scoreboard "
                 "stalls 6.3 per issue; DRAM 13 %, FMA/ALU pipes 38-41 % (ncu capture on dx=0.0138)")
MIN_TIMED_SOLVER_STEPS = 200


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--chunk", type=int, default=0,
                    help="solver steps per bench step (0: the least that makes K bench steps "
                         f"cover {MIN_TIMED_SOLVER_STEPS} solver steps)")
    ap.add_argument("--ref-dx", type=float, default=0.0276,
                    help="lattice spacing of the CPU reference rung")
    ap.add_argument("--ref-sample-steps", type=int, default=3,
                    help="solver steps of the reference's CPU code timed for cpu_baseline")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--dx", type=float, default=0.0069)
    ap.add_argument("--shift-every", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--skin", type=float, default=0.0,
                    help="with --no-tune: the list skin in h (0: the configuration's 0.25)")
    ap.add_argument("--block", type=int, default=0, help="with --no-tune: pair-kernel block size (0: 128)")
    ap.add_argument("--batch", type=int, default=0, help="with --no-tune: batch depth 4, 8 or 16 (0: 4)")
    ap.add_argument("--cpu-sample-steps", type=int, default=6)
    ap.add_argument("--ensemble-cases", type=int, default=256)
    ap.add_argument("--ensemble-steps", type=int, default=100)
    ap.add_argument("--plain-steps", type=int, default=100)
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-time-scale", type=float, default=0.05)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-tight-gb", type=float, default=4.0,
                    help="a second served run under this HBM budget, small enough that admissions "
                         "wait for retirements (0: none)")
    ap.add_argument("--dplus-dx", type=float, default=0.0138,
                    help="lattice spacing of the 3-D delta-plus leg (0: no leg)")
    ap.add_argument("--dplus-steps", type=int, default=20)
    ap.add_argument("--shear-n", type=int, default=64)
    ap.add_argument("--shear-steps", type=int, default=2000)
    ap.add_argument("--csf3-radius", type=int, default=40, help="column radius in dx (0: no 3-D CSF leg)")
    ap.add_argument("--csf3-length", type=int, default=200, help="column period in dx")
    ap.add_argument("--tvc-n", type=int, default=100, help="fluid block edge in dx (0: no TVC leg)")
    ap.add_argument("--rhs2d-dx", type=float, default=0.0014,
                    help="lattice spacing of the 2-D rhs leg's 1 x 2 m column (0: no rhs leg)")
    ap.add_argument("--ckpt-steps", type=int, default=200, help="steps of the checkpoint leg (0: no leg)")
    ap.add_argument("--ckpt-every", type=int, default=100, help="checkpoint interval of the checkpoint leg")
    return ap.parse_args()


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest value over all ranks (every rank calls it, in the same order)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def whole_job_rate(units_per_rank: int, steps: int, world: int, seconds: float) -> float:
    """Units processed by all ranks divided by the (max-over-ranks) time."""
    return units_per_rank * steps * world / seconds


def driver_peaks():
    """HBM GB/s and bf16 TF/s measured on this pool (MEASURED_PEAKS.json), if present."""
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text())
    return None


def probe_peaks(dev):
    """The FP32 FMA rate (scalar and packed FP32x2 chains, the larger) and the
    device copy bandwidth of this GPU, each the best of 3 CUDA-event-timed
    launches of the library's probe kernels after a warm-up launch."""
    import torch
    from tensorsph_b200 import _lib
    L = _lib.lib()
    s = torch.cuda.current_stream(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, threads, iters = sms * 8, 256, 4096
    out = torch.empty(blocks * threads, dtype=torch.float32, device=dev)

    def best_ms(launch):
        best = None
        for rep in range(4):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            launch()
            b.record(s)
            b.synchronize()
            if rep:
                ms = a.elapsed_time(b)
                best = ms if best is None else min(best, ms)
        return best

    fma = {}
    for packed in (0, 1):
        ms = best_ms(lambda: _lib.check(L.tsph_probe_fma(out.data_ptr(), blocks, threads, iters, packed,
                                                         s.cuda_stream), "tsph_probe_fma"))
        fma["packed" if packed else "scalar"] = (L.tsph_probe_fma_flops(blocks, threads, iters, packed)
                                                 / (ms / 1e3) / 1e12)
    nbytes = 2 << 30
    src = torch.ones(nbytes, dtype=torch.uint8, device=dev)
    dst = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    ms = best_ms(lambda: _lib.check(L.tsph_probe_copy(src.data_ptr(), dst.data_ptr(), nbytes, sms * 16,
                                                      s.cuda_stream), "tsph_probe_copy"))
    del src, dst
    torch.cuda.empty_cache()
    return {"fp32_tflops": max(fma.values()), "fp32_scalar_tflops": fma["scalar"],
            "fp32_packed_tflops": fma["packed"], "copy_gbs": 2 * nbytes / (ms / 1e3) / 1e9,
            "probe": f"FMA: {blocks}x{threads} threads x 8 chains x {iters}; copy: 2 GiB read + 2 GiB write"}


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [r.split(",") for r in out.strip().splitlines() if r.strip()]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for name, val in zip(names, r[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


REF_PATH = ROOT / "baseline" / "_ref"


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_available() -> bool:
    return (REF_PATH / "tensorsph" / "dam_break_3d.py").exists()


def reference_loop(dx, steps, warmup, shift_every, threads=None):
    """The reference's own CPU code on one rung of the headline case: the
    obstacle loop of kleefsman_obstacle_3d.py:644-706 (PairListCache.get,
    rhs_3d with the wall force, Euler, apply_boundary_3d, clamp_out_of_obstacle)
    with the shifting hook of dam_break.py:424-433 (shift_positions every
    ``shift_every`` steps from the second step on), in the reference's default
    dtype (FP32), torch on ``threads`` host threads (all usable cores).  The
    tank and obstacle are this case's geometry, built with the reference's own
    lattice builders; validate_case is skipped because the geometry is not
    Kleefsman's (kleefsman_obstacle_3d.py:129-147).  Returns fluid
    particle-updates/s over ``steps`` timed steps after ``warmup`` steps."""
    if str(REF_PATH) not in sys.path:
        sys.path.insert(0, str(REF_PATH))
    import torch
    from tensorsph.dam_break_3d import DamBreak3DConfig, apply_boundary_3d, make_column_3d, rhs_3d, wall_lattice_3d
    from tensorsph.kleefsman_obstacle_3d import clamp_out_of_obstacle, obstacle_lattice_3d
    from tensorsph.neighbor_search import PairListCache
    from tensorsph.particle_shifting import shift_positions
    threads = threads or max(1, len(os.sched_getaffinity(0)))
    torch.set_num_threads(threads)
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 0.55)
    h = 1.3 * dx
    cfg = DamBreak3DConfig(dx=dx, pool_width=3.2, tank_depth=1.0, tank_height=1.0, column_width=1.2,
                           column_depth=1.0, column_height=0.55, wall_layers=3, density_diffusion=0.1,
                           sound_speed=c0, viscosity=1.0e-6, dt=0.25 * h / c0, max_courant=0.25, steps=5000)

    class ObstacleBox:
        """The obstacle fields clamp_out_of_obstacle and obstacle_lattice_3d read."""
        obstacle_x, obstacle_height, obstacle_z = 3.2 - 0.744 - 0.08, 0.16, 0.3

        def __init__(self):
            self.dx = dx

        def obstacle_x1(self):
            return self.obstacle_x + 0.16

        def obstacle_z1(self):
            return 0.7

    box = ObstacleBox()
    dev = torch.device("cpu")
    pos, mass = make_column_3d(cfg, dev)
    wall = torch.cat((wall_lattice_3d(cfg, dev, top=cfg.tank_top()),
                      obstacle_lattice_3d(box, dev).to(pos.dtype)))
    vel = torch.zeros_like(pos)
    n = pos.shape[0]
    cache = PairListCache(2.0 * h, cfg.pair_skin_factor * h, fluid_count=n)
    all_pos = torch.cat((pos, wall))
    t0 = None
    for step in range(warmup + steps):
        if step == warmup:
            t0 = time.perf_counter()
        all_pos[:n] = pos
        pairs, _ = cache.get(all_pos)
        rho, _, acc, _ = rhs_3d(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt, return_wall_force=True)
        speed = float(torch.linalg.vector_norm(vel, dim=-1).max())
        vel = vel + cfg.dt * acc
        pos = pos + cfg.dt * vel
        apply_boundary_3d(pos, vel, cfg, top=cfg.tank_top())
        clamp_out_of_obstacle(pos, vel, box)
        if shift_every and step > 0 and step % shift_every == 0:
            pos = shift_positions(pos, mass / rho, h, dt=cfg.dt, v_ref=max(speed, 0.05 * c0))
    elapsed = time.perf_counter() - t0
    return {"value": n * steps / elapsed, "fluid": n, "seconds": elapsed, "cores": threads,
            "rebuilds": cache.rebuilds, "torch": torch.__version__, "cpu": cpu_model(),
            "dtype": str(pos.dtype).replace("torch.", "")}


def oracle_port_and_errors(dx, dev, shift_every, tuning, max_lead=8000):
    """The oracle port (numpy FP64, one core) on one rung of the headline
    case, timed, and the engine's FP32-pair run of the same rung against it,
    field by field (the FP64 run each reported field carries its error
    against).  Two phases: from rest (3 steps), and the impact on the obstacle
    (the engine runs from rest until the surge loads the obstacle, at most
    ``max_lead`` steps; from its state both take 2 steps).  Errors: density /
    rho0, pressure / B, acceleration / its largest value, obstacle force / its
    largest value, front / dx."""
    import numpy as np
    from dataclasses import replace
    from oracle import dam3d
    from tensorsph_b200.engine import DamBreak3DEngine, obstacle_case
    cfg, ob = obstacle_case(dx=dx)
    if tuning is not None:
        cfg = replace(cfg, pair_skin_factor=tuning["best"]["skin_factor"])
    x, m, w, n_ob = DamBreak3DEngine.build_host_state(cfg, ob)
    bulk = cfg.rho0 * cfg.sound_speed ** 2 / cfg.gamma
    out = {"rung": f"dx={dx:g} ({x.shape[0]} fluid + {w.shape[0]} wall)"}
    port_steps, port_time = 0, 0.0

    def fields(eng, recs, first, count, k_state):
        diag = eng.diagnostics(first, count).cpu().numpy()
        _, _, erho, ep = (t.cpu().numpy() for t in eng.state())
        r = recs[k_state]
        e = {"density": float(np.abs(erho - r["rho"]).max()) / cfg.rho0,
             "pressure": float(np.abs(ep - r["p"]).max()) / bulk,
             "rho_max": max(abs(diag[k, 0] - recs[k]["rho"].max()) for k in range(count)) / cfg.rho0,
             "front": max(abs(diag[k, 2] - recs[k]["front"]) for k in range(count)) / cfg.dx}
        fmax = max(float(np.abs(rr["force"]).max()) for rr in recs)
        if fmax > 0:
            e["obstacle_force"] = max(float(np.abs(diag[k, 3:6] - recs[k]["force"]).max())
                                      for k in range(count)) / fmax
            e["obstacle_force_N"] = fmax
        return e

    # from rest
    t0 = time.perf_counter()
    recs, _, _ = dam3d.run(cfg, ob, x.numpy(), m.numpy(), w.numpy(), n_ob, 3, shift_every=shift_every)
    port_time += time.perf_counter() - t0
    port_steps += 3
    eng = DamBreak3DEngine(cfg, obstacle=ob, shift_every=shift_every, host_state=(x, m, w, n_ob),
                           diag_ring=64, device=dev)
    eng.step(1)
    _, ev, erho, ep = (t.cpu().numpy() for t in eng.state())
    v1 = cfg.dt * recs[0]["acc"]
    rest = {"density": float(np.abs(erho - recs[0]["rho"]).max()) / cfg.rho0,
            "pressure": float(np.abs(ep - recs[0]["p"]).max()) / bulk,
            "acceleration": float(np.abs(ev - v1).max()) / float(np.abs(v1).max()),
            "acceleration_yardstick": "max |a| of the step (hydrostatic cancellation)"}
    eng.step(2)
    rest.update({f"{k}_step3": v for k, v in fields(eng, recs, 0, 3, 2).items()})
    eng.close()
    out["from_rest"] = rest
    # impact on the obstacle
    eng = DamBreak3DEngine(cfg, obstacle=ob, shift_every=shift_every, host_state=(x, m, w, n_ob),
                           diag_ring=max_lead + 64, device=dev)
    lead, f_lead = 0, np.zeros(3)
    while np.abs(f_lead).max() < 1.0 and lead < max_lead:
        eng.step(250)
        lead += 250
        f_lead = eng.diagnostics(lead - 1, 1).cpu().numpy()[0, 3:6]
    eng.step(50)
    lead += 50
    xs, vs, _, _ = (t.cpu() for t in eng.state())
    eng.close()
    t0 = time.perf_counter()
    recs, _, _ = dam3d.run(cfg, ob, xs.numpy(), m.numpy(), w.numpy(), n_ob, 2, shift_every=shift_every,
                           v0=vs.numpy(), first_step=lead)
    port_time += time.perf_counter() - t0
    port_steps += 2
    eng = DamBreak3DEngine(cfg, obstacle=ob, shift_every=shift_every, host_state=(xs, m, w, n_ob),
                           velocity=vs, first_step=lead, diag_ring=64, device=dev)
    eng.step(2)
    impact = fields(eng, recs, lead, 2, 1)
    impact["after_steps"] = lead
    eng.close()
    out["impact"] = impact
    out["port"] = {"value": x.shape[0] * port_steps / port_time, "unit": "fluid particle-updates/s",
                   "cores": 1, "kind": "port", "seconds": port_time,
                   "sample": f"{port_steps} FP64 steps of the oracle loop on the {out['rung']} rung"}
    return out


def ensemble_leg(args, dev):
    """Batched droplet ensemble vs the same cases one at a time (both device
    timed); block size and skin chosen by the autotuner on a 32-case sample."""
    from tensorsph_b200 import ensemble as en
    draws = en.draw_ensemble(args.ensemble_cases, seed=0)
    tune = en.autotune(draws[:32], steps=20, warmup=5, device=dev)
    best = tune["best"]
    specs = en.ensemble_specs(draws, skin_factor=best["skin_factor"])
    batched = en.run_batched(specs, args.ensemble_steps, block=best["block"], batch=best["batch"],
                             device=dev)
    # the one-at-a-time arm tuned the same way, on one case alone
    tune_plain = en.autotune(draws[:1], steps=20, warmup=5, device=dev)
    bp = tune_plain["best"]
    plain = en.run_plain(en.ensemble_specs(draws, skin_factor=bp["skin_factor"]), args.plain_steps,
                         block=bp["block"], batch=bp["batch"], device=dev)
    return {"workload": f"{len(specs)} independent 2-D droplet impacts (R~U[0.02,0.08] m, dx=R/20, "
                        "depth~U[2R,6R], width 8R, U~U[1,5] m/s, seed 0), CSF sigma=0.0728 N/m",
            "fluid_particles": batched["fluid"],
            "batched_updates_per_s": batched["updates_per_s"],
            "batched_ms_per_step": 1e3 * batched["seconds"] / batched["steps"],
            "plain_updates_per_s": plain["updates_per_s"],
            "speedup_vs_plain": batched["updates_per_s"] / plain["updates_per_s"],
            "kernels_per_step": batched["kernels_per_step"], "failed_cases": batched["failed_cases"],
            "autotune": {"best": best, "trials": len(tune["trials"]), "cached": tune.get("cached"),
                         "plain_best": bp},
            "steps": {"batched": batched["steps"], "plain_per_case": plain["steps"]}}


def serving_leg(args, dev):
    """Continuous-batching server vs serial single-case runs of one seeded
    stream, at the configured budget and, with ``--serve-tight-gb``, again
    under a budget small enough that admissions wait for retirements
    (admission by HBM footprint)."""
    import torch
    from tensorsph_b200 import serving as sv

    def stream():
        return sv.request_stream(args.serve_requests, rate=20.0, seed=0, time_scale=args.serve_time_scale)

    out = {"workload": f"{args.serve_requests} requests, Poisson 20/s (seed 0), types "
                       f"{list(sv.CASE_TYPES)}, fluid log-uniform [1e3, 2e6], simulated time "
                       f"U[0.1, 1.0] s x {args.serve_time_scale:g}",
           "time_scale": args.serve_time_scale}
    serial = sv.run_serial(stream(), device=dev)
    out["serial"] = {"updates_per_s": serial["updates_per_s"], "wall_s": serial["wall_s"],
                     "latency_s": serial["latency_s"]}
    for name, budget in (("batched", args.serve_budget_gb), ("batched_tight", args.serve_tight_gb)):
        if budget <= 0:
            continue
        srv = sv.Server(budget_bytes=budget * 1e9, device=dev)
        served = srv.serve(stream())
        engine_gb = srv.engine_bytes / 1e9
        srv.close()
        torch.cuda.empty_cache()
        out[name] = {"budget_gb": budget, "engine_gb": engine_gb,
                     "updates_per_s": served["updates_per_s"], "wall_s": served["wall_s"],
                     "latency_s": served["latency_s"], "admissions_blocked": served["admissions_blocked"],
                     "graph_instantiations": served["graph_instantiations"],
                     "graph_updates": served["graph_updates"], "engine_steps": served["engine_steps"],
                     "throughput_vs_serial": served["updates_per_s"] / serial["updates_per_s"]}
    out["throughput_vs_serial"] = out["batched"]["throughput_vs_serial"]
    return out


def delta_plus_leg(args, dev):
    """The 3-D dam break with the obstacle advanced by delta-plus steps
    (delta_plus_step3 through threed/delta_plus3.py, FP32): device time per
    step, pair cache included, with the density deviation and the front."""
    import torch
    from tensorsph_b200.engine import obstacle_case
    from tensorsph_b200.threed.delta_plus3 import delta_plus_case_3d, run_delta_plus_3d
    cfg, ob = obstacle_case(dx=args.dplus_dx)
    host = delta_plus_case_3d(cfg, ob, torch.float32)
    run_delta_plus_3d(cfg, 2, obstacle=ob, dtype=torch.float32, host_state=host, device=dev)
    run = run_delta_plus_3d(cfg, args.dplus_steps, obstacle=ob, dtype=torch.float32, host_state=host, device=dev)
    return {"workload": f"3-D dam break with the box obstacle, delta-plus (h = 2 dx, Wendland C2, psi "
                        f"diffusion 0.1, alpha 0.02, 4 station layers), dx={args.dplus_dx:g}, FP32, "
                        f"{args.dplus_steps} steps from the hydrostatic start",
            "fluid_particles": run.n_fluid, "wall_stations": run.n_wall,
            "ms_per_step": 1e3 * run.seconds / run.steps,
            "fluid_particles_per_s": run.n_fluid * run.steps / run.seconds,
            "pair_rebuilds": run.rebuilds, "max_density_deviation": max(run.density_deviation),
            "max_shift_over_dx": run.max_shift_over_dx, "front": [run.front[0], run.front[-1]]}


def shear_leg(args, dev):
    """Triply periodic shear decay u_x = 1e-3 sin(2 pi z), n^3 jittered lattice,
    nu = 1e-2, c0 = 1: the same driver with FP32 (compensated) pair arithmetic on
    an FP64 state ("fp32"), everything in FP32 ("fp32_state_fp32") and all FP64;
    decay rates against nu k^2 and the FP32 density fields against FP64."""
    import torch
    from tensorsph_b200.threed.shear import run_shear_decay
    out = {"workload": f"{args.shear_n}^3 periodic shear decay, u_x=1e-3 sin(2 pi z), nu=1e-2, "
                       f"c0=1, h=1.3dx, jitter 0.01dx (seed 0), {args.shear_steps} KDK steps"}
    runs = {}
    for name, dtype, state in (("fp32", torch.float32, torch.float64),
                               ("fp32_state_fp32", torch.float32, torch.float32),
                               ("fp64", torch.float64, torch.float64)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = run_shear_decay(n=args.shear_n, steps=args.shear_steps, dtype=dtype, state_dtype=state,
                            device=dev)
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        runs[name] = r
        out[name] = {"fit_rate": r.fit_rate, "analytic_rate": r.analytic_rate,
                     "rate_rel_error": r.rate_error, "pair_rebuilds": r.pair_rebuilds,
                     "ms_per_step": 1e3 * wall / args.shear_steps,
                     "updates_per_s": args.shear_n ** 3 * args.shear_steps / wall,
                     "momentum_final_over_scale": r.diagnostics[-1]["momentum_magnitude"]
                     / r.momentum_scale}
    b = runs["fp64"]
    for name in ("fp32", "fp32_state_fp32"):
        a = runs[name]
        out[name]["rate_rel_diff_vs_fp64"] = (a.fit_rate - b.fit_rate) / b.fit_rate
        out[name]["density_max_abs_diff_over_rho0"] = float(
            (a.final_density.double() - b.final_density).abs().max()) / 1000.0
    return out


def _column(radius, length, dx, seed, device):
    """A liquid column along z, periodic in a box of (2R + 8 dx)^2 x L: the
    lattice points with r <= R, jittered by 0.05 dx (seeded)."""
    import torch
    side = 2 * radius + 8
    box = [side * dx, side * dx, length * dx]
    g = torch.Generator().manual_seed(seed)
    a = (torch.arange(side, dtype=torch.float64) + 0.5) * dx
    X, Y = torch.meshgrid(a, a, indexing="ij")
    keep = (X - 0.5 * box[0]) ** 2 + (Y - 0.5 * box[1]) ** 2 <= (radius * dx) ** 2
    xy = torch.stack((X[keep], Y[keep]), -1)
    z = (torch.arange(length, dtype=torch.float64) + 0.5) * dx
    pos = torch.cat((xy.repeat(length, 1), z.repeat_interleave(xy.shape[0])[:, None]), 1)
    pos = pos + 0.05 * dx * (2.0 * torch.rand(pos.shape, generator=g, dtype=torch.float64) - 1.0)
    pos = torch.remainder(pos, torch.tensor(box, dtype=torch.float64))
    return pos.to(device), box


def csf3_leg(args, dev):
    """3-D CSF surface tension (csf_fields3 "mls" + surface_tension_acceleration3)
    on a periodic liquid column (the Rayleigh-Plateau geometry): device time of
    the drop-in call -- pair rows, fields and acceleration -- per particle, with
    the oracle's CPU rate on a small column beside it."""
    import numpy as np
    import torch
    from tensorsph_b200.threed.csf3 import csf_fields3, surface_tension_acceleration3
    from tensorsph_b200.threed.neighbors3 import periodic_pairs
    dx, h = 1e-3, 1.3e-3
    pos, box = _column(args.csf3_radius, args.csf3_length, dx, 7, dev)
    n = pos.shape[0]
    mass = torch.full((n,), 1000.0 * dx ** 3, dtype=torch.float64, device=dev)
    rho = torch.full((n,), 1000.0, dtype=torch.float64, device=dev)
    pairs = periodic_pairs(pos, box, 2.0 * h)

    def call():
        st = csf_fields3(pos, mass, h, pairs, rho0=1000.0, box=box)
        return st, surface_tension_acceleration3(st, rho, 0.0728)

    for _ in range(2):
        st, acc = call()
    reps = 5
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    start.record()
    for _ in range(reps):
        st, acc = call()
    stop.record()
    torch.cuda.synchronize(dev)
    ms = start.elapsed_time(stop) / reps
    shell = st.surface_mask(0.3) & st.valid
    off = pos[shell, :2] - torch.tensor(box[:2], dtype=torch.float64, device=dev) * 0.5
    radial = off / off.norm(dim=1, keepdim=True)
    a = acc[shell]
    cos = float(((a[:, :2] * radial).sum(1) / a.norm(dim=1).clamp_min(1e-30)).mean())
    # CPU: the oracle on a small column (R = 8 dx, period 24 dx)
    from oracle import csf3 as oc
    from oracle.neighbors import periodic_pairs as np_periodic_pairs
    small, sbox = _column(8, 24, dx, 7, "cpu")
    sp = small.numpy()
    smass = np.full(sp.shape[0], 1000.0 * dx ** 3)
    t0 = time.perf_counter()
    spairs = np_periodic_pairs(sp, np.asarray(sbox), 2.0 * h)
    sst = oc.csf_fields3(sp, smass, h, spairs, rho0=1000.0, box=np.asarray(sbox))
    oc.surface_tension_acceleration3(sst, np.full(sp.shape[0], 1000.0), 0.0728)
    t_cpu = time.perf_counter() - t0
    return {"workload": f"periodic liquid column R={args.csf3_radius} dx, period {args.csf3_length} dx, "
                        "dx=1 mm, h=1.3 dx, jitter 0.05 dx (seed 7), FP64",
            "particles": n, "pairs": int(pairs.shape[0]), "ms_per_call": ms,
            "particles_per_s": n / (ms / 1e3), "shell_force_cos_to_axis": cos,
            "valid_fraction": float(st.valid.double().mean()),
            "cpu_oracle": {"particles_per_s": sp.shape[0] / t_cpu, "particles": sp.shape[0],
                           "cores": 1, "seconds": t_cpu,
                           "sample": "R=8 dx, period 24 dx column: pairs + fields + acceleration"}}


def tvc_leg(args, dev):
    """Transport-velocity correction (transport_velocity_correction, no limiter)
    on a jittered n^3 fluid block over three wall layers: device time of the
    drop-in call -- pair rows, gradient integral and displacement -- per fluid
    particle, with the oracle's CPU rate on a small block beside it."""
    import numpy as np
    import torch
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    from tensorsph_b200.transport_velocity_correction import transport_velocity_correction

    def block(n, seed, device):
        dx = 0.002
        g = torch.Generator().manual_seed(seed)
        ax = (torch.arange(n, dtype=torch.float64) + 0.5) * dx
        X, Y, Z = torch.meshgrid(ax, ax, ax, indexing="ij")
        fluid = torch.stack((X.reshape(-1), Y.reshape(-1), Z.reshape(-1)), 1)
        fluid = fluid + 0.08 * dx * torch.randn(fluid.shape, generator=g, dtype=torch.float64)
        wx = (torch.arange(-3, n + 3, dtype=torch.float64) + 0.5) * dx
        wl = (torch.arange(-3, 0, dtype=torch.float64) + 0.5) * dx
        WX, WY, WZ = torch.meshgrid(wx, wl, wx, indexing="ij")
        wall = torch.stack((WX.reshape(-1), WY.reshape(-1), WZ.reshape(-1)), 1)
        pos = torch.cat((fluid, wall)).to(device)
        vol = torch.full((pos.shape[0],), dx ** 3, dtype=torch.float64, device=device)
        return pos, vol, wall.shape[0], 1.3 * dx

    pos, vol, nw, h = block(args.tvc_n, 11, dev)
    pairs = cell_linked_pairs(pos, 2.0 * h)
    call = lambda: transport_velocity_correction(pos, vol, h, pairs=pairs, wall_count=nw, max_shift=0.05 * h)
    for _ in range(2):
        res = call()
    reps = 5
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    start.record()
    for _ in range(reps):
        res = call()
    stop.record()
    torch.cuda.synchronize(dev)
    ms = start.elapsed_time(stop) / reps
    nf = pos.shape[0] - nw
    from oracle import tvc as otv
    from oracle.neighbors import cell_linked_pairs as np_pairs
    spos, svol, snw, sh = block(16, 11, "cpu")
    sp, sv = spos.numpy(), svol.numpy()
    t0 = time.perf_counter()
    otv.transport_velocity_correction(sp, sv, sh, np_pairs(sp, 2.0 * sh), wall_count=snw, max_shift=0.05 * sh)
    t_cpu = time.perf_counter() - t0
    return {"workload": f"{args.tvc_n}^3 jittered fluid block (0.08 dx, seed 11) over 3 wall layers, dx=2 mm, "
                        "h=1.3 dx, no limiter, max_shift 0.05 h, FP64",
            "fluid_particles": nf, "wall_particles": nw, "pairs": int(pairs.shape[0]), "ms_per_call": ms,
            "fluid_particles_per_s": nf / (ms / 1e3), "clipped_fraction": res.clipped,
            "max_shift_over_h": res.max_shift / h,
            "cpu_oracle": {"fluid_particles_per_s": (spos.shape[0] - snw) / t_cpu,
                           "fluid_particles": spos.shape[0] - snw, "cores": 1, "seconds": t_cpu,
                           "sample": "16^3 block: pairs + gradient integral + displacement"}}


def rhs2d_leg(args, dev):
    """The 2-D rhs drop-in (droplet_impact.rhs, droplet_impact.py:810-1228) on
    a jittered resting dam-break column with three wall layers, FP32 as the
    reference runs it: device time of one call with the step's pair list
    given -- gather rows, density, Molteni diffusion, Tait, Adami walls,
    pressure and viscous force -- per fluid particle, with the oracle's CPU
    rate on a small column beside it."""
    import numpy as np
    import torch
    from oracle import pairpass as op
    from oracle.neighbors import cell_linked_pairs as np_pairs
    from tensorsph_b200.dam_break import DamBreakConfig, make_column
    from tensorsph_b200.droplet_impact import rhs, wall_lattice
    from tensorsph_b200.neighbor_search import cell_linked_pairs

    def state(dx, device):
        c0 = 62.6
        cfg = DamBreakConfig(dx=dx, column_width=1.0, column_height=2.0, pool_width=4.0, tank_height=3.0,
                             sound_speed=c0, viscosity=1e-6, density_diffusion=0.1, max_courant=0.25,
                             dt=0.25 * 1.3 * dx / c0, wall_layers=3)
        pos, mass = make_column(cfg, "cpu")
        wall = wall_lattice(cfg, "cpu", top=cfg.tank_top())
        g = torch.Generator().manual_seed(5)
        pos = pos + (0.05 * dx * torch.randn(pos.shape, generator=g, dtype=torch.float64)).to(pos.dtype)
        return cfg, pos.to(device), mass.to(device), wall.to(device)

    saved = torch.get_default_dtype()
    torch.set_default_dtype(torch.float32)
    try:
        cfg, pos, mass, wall = state(args.rhs2d_dx, dev)
        h = cfg.h_factor * cfg.dx
        allpos = torch.cat((pos, wall))
        pairs = cell_linked_pairs(allpos, 2.0 * h)
        pairs = pairs[(pairs[:, 0] < pos.shape[0]) | (pairs[:, 1] < pos.shape[0])]
        vel = torch.zeros_like(pos)
        call = lambda: rhs(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt)  # noqa: E731
        for _ in range(2):
            rho, p, acc = call()
        reps = 5
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        start.record()
        for _ in range(reps):
            rho, p, acc = call()
        stop.record()
        torch.cuda.synchronize(dev)
        ms = start.elapsed_time(stop) / reps
        scfg, spos, smass, swall = state(0.02, "cpu")
        sp, sw = spos.numpy(), swall.numpy()
        sall = np.concatenate((sp, sw))
        t0 = time.perf_counter()
        spairs = np_pairs(sall, 2.0 * scfg.h_factor * scfg.dx)
        spairs = spairs[(spairs[:, 0] < sp.shape[0]) | (spairs[:, 1] < sp.shape[0])]
        op.rhs(sp, np.zeros_like(sp), smass.numpy(), scfg, pairs=spairs, wall=sw, dt=scfg.dt)
        t_cpu = time.perf_counter() - t0
        # the timed path (FP32) on the oracle's column against the FP64 oracle
        d_rho, d_p, d_acc = (t.double().cpu().numpy() for t in rhs(
            spos.to(dev), torch.zeros_like(spos).to(dev), smass.to(dev), scfg,
            pairs=torch.from_numpy(spairs).to(dev), wall=swall.to(dev), dt=scfg.dt))
        f64 = np.float64
        o_rho, o_p, o_acc = op.rhs(sp.astype(f64), np.zeros(sp.shape, f64), smass.numpy().astype(f64), scfg,
                                   pairs=spairs, wall=sw.astype(f64), dt=scfg.dt)
        bulk = scfg.rho0 * scfg.sound_speed ** 2 / scfg.gamma
        at = int(np.argmax(o_rho))
        errors = {"rho_over_rho0": float(np.abs(d_rho - o_rho).max() / scfg.rho0),
                  "p_over_B": float(np.abs(d_p - o_p).max() / bulk),
                  "acc_over_max_acc": float(np.abs(d_acc - o_acc).max() / np.abs(o_acc).max()),
                  "oracle_rho_max_over_rho0": float(o_rho[at] / scfg.rho0),
                  "oracle_rho_max_at": [float(v) for v in sp[at]],
                  "sample": "dx=0.02 column (the CPU rate's), device FP32 vs oracle FP64"}
    finally:
        torch.set_default_dtype(saved)
    n = pos.shape[0]
    return {"workload": f"resting 1.0 x 2.0 m column, dx={args.rhs2d_dx} m, jitter 0.05 dx (seed 5), 3 wall layers, "
                        "c0=62.6, Molteni delta=0.1, FP32, pair list given",
            "fluid_particles": n, "wall_particles": int(wall.shape[0]), "pairs": int(pairs.shape[0]),
            "ms_per_call": ms, "fluid_particles_per_s": n / (ms / 1e3),
            "rho_max_over_rho0": float(rho.max()) / cfg.rho0,
            "errors_vs_fp64": errors,
            "cpu_oracle": {"fluid_particles_per_s": sp.shape[0] / t_cpu, "fluid_particles": sp.shape[0],
                           "cores": 1, "seconds": t_cpu,
                           "sample": "dx=0.02 column: pairs + density, diffusion, walls, force"}}


def checkpoint_leg(args, dev, cfg, obstacle, host, tuning):
    """The headline run with crash-safe checkpoints (the obstacle case's
    format, kleefsman_obstacle_3d.py:477-546) every ``--ckpt-every`` steps,
    against the same steps without: device time of the step loop on the
    engine's stream (the state read kernel is on it; the copies to pinned
    memory are on a side stream and the file write on a thread), the wall
    time of the loop, and each write's time on its thread."""
    import shutil
    import tempfile

    import torch
    from tensorsph_b200.checkpoint import CheckpointWriter
    from tensorsph_b200.engine import DamBreak3DEngine, _DeviceRecord, _elapsed_after, _sample_steps
    steps, every, warm = args.ckpt_steps, max(args.ckpt_every, 1), 3
    folder = tempfile.mkdtemp(prefix="tsph_ckpt_")
    path = os.path.join(folder, "state.pt")
    out = {"steps": steps, "every": every}
    try:
        for mode in ("plain", "checkpoint"):
            eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=args.shift_every, host_state=host,
                                   diag_ring=steps + warm + 16, device=dev)
            if tuning is not None:
                eng.set_block(tuning["best"]["block"])
                eng.set_batch(tuning["best"]["batch"])
            eng.step(warm)
            torch.cuda.synchronize(dev)
            writer = None
            if mode == "checkpoint":
                writer = CheckpointWriter(eng, eng.case_id, path, cfg, obstacle=obstacle)
                record = _DeviceRecord(cfg, _sample_steps(cfg.steps, cfg.output_every, cfg.dt), 0, None,
                                       eng.n_fluid, eng.initial_pe)
                after = _elapsed_after(cfg.steps, cfg.dt)
            start = torch.cuda.Event(enable_timing=True)
            stop = torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            start.record(eng.stream)
            done = warm
            for _ in range(steps // every):
                eng.step(every)
                done += every
                if writer is not None:
                    k = done - 1
                    writer.take(k, after[k + 1], 0, k + 1, lambda rows, k=k: record.payload(rows, k))
            stop.record(eng.stream)
            torch.cuda.synchronize(dev)
            loop_s = time.perf_counter() - t0
            row = {"device_ms_per_step": start.elapsed_time(stop) / (done - warm),
                   "wall_ms_per_step": loop_s * 1e3 / (done - warm)}
            if writer is not None:
                writer.close()
                row.update(written=writer.written, write_s=writer.write_seconds,
                           file_bytes=os.path.getsize(path),
                           drain_s=time.perf_counter() - t0 - loop_s)
            out[mode] = row
            eng.close()
            del eng
            torch.cuda.empty_cache()
        p, c = out["plain"], out["checkpoint"]
        out["device_overhead"] = c["device_ms_per_step"] / p["device_ms_per_step"] - 1.0
        out["wall_overhead"] = c["wall_ms_per_step"] / p["wall_ms_per_step"] - 1.0
    finally:
        shutil.rmtree(folder, ignore_errors=True)
    return out


def workload_config(args) -> dict:
    """The workload both arms' lines name."""
    return {"workload": "3-D dam break with box obstacle: 1.2x1.0x0.55 m fluid in a 3.2x1.0x1.0 m tank, "
                        f"obstacle 0.16x0.16x0.4 m, dx={args.dx:g}",
            "shift_every": args.shift_every, "density_diffusion": 0.1}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    chunk = args.chunk if args.chunk > 0 else max(1, math.ceil(MIN_TIMED_SOLVER_STEPS / max(args.steps, 1)))

    if args.impl == "reference":
        if rank != 0:
            return
        workload = (f"each step one solver step of the reference's own CPU loop on the dx={args.ref_dx:g} "
                    "rung of the same case (a full-size step takes ~40 s on the host)")
        if reference_available():
            r = reference_loop(args.ref_dx, args.steps, max(args.warmup, 1), args.shift_every)
            kind = "reference"
            sample = (f"{args.steps} solver steps after {max(args.warmup, 1)} warm-up steps of the "
                      f"dx={args.ref_dx:g} rung ({r['fluid']} fluid), tensorsph from baseline/_ref, "
                      f"torch {r['torch']} {r['dtype']} on {r['cores']} threads ({r['cpu']}), "
                      f"{r['seconds']:.1f} s, {r['rebuilds']} list builds")
            value, cores, dtype = r["value"], r["cores"], r["dtype"]
        else:
            # the reference is not installed: its algorithm, restated as the
            # oracle port (numpy FP64, one core)
            from tensorsph_b200.engine import DamBreak3DEngine, obstacle_case
            from oracle import dam3d
            cfg, ob = obstacle_case(dx=args.ref_dx)
            x, m, w, n_ob = DamBreak3DEngine.build_host_state(cfg, ob)
            k = max(args.steps // 10, 2)
            t0 = time.perf_counter()
            dam3d.run(cfg, ob, x.numpy(), m.numpy(), w.numpy(), n_ob, k, shift_every=args.shift_every,
                      record=False)
            el = time.perf_counter() - t0
            value, cores, dtype, kind = x.shape[0] * k / el, 1, "f64", "port"
            sample = f"{k} steps of the oracle port on the dx={args.ref_dx:g} rung, {el:.1f} s"
        line = {"metric": "particle-updates/s", "value": value, "unit": "fluid particle-updates/s",
                "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded lattice)",
                "config": {**workload_config(args), "reference_sample": workload},
                "cpu_baseline": {"value": value, "unit": "fluid particle-updates/s", "cores": cores,
                                 "kind": kind, "sample": sample},
                "e2e": {"value": value, "unit": "fluid particle-updates/s",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from tensorsph_b200.engine import DamBreak3DEngine, obstacle_case

    cfg, obstacle = obstacle_case(dx=args.dx)
    host = DamBreak3DEngine.build_host_state(cfg, obstacle)
    tuning = None
    if not args.no_tune:
        # untimed: pick the list skin, block size and batch depth on this case
        from dataclasses import replace
        from tensorsph_b200.engine import tune_single_case
        tuning = tune_single_case(cfg, obstacle=obstacle, shift_every=args.shift_every,
                                  host_state=host, device=dev)
        cfg = replace(cfg, pair_skin_factor=tuning["best"]["skin_factor"])
    elif args.skin or args.block or args.batch:
        # a fixed choice (for profiling the tuned configuration without tuning)
        from dataclasses import replace
        tuning = {"best": {"skin_factor": args.skin or cfg.pair_skin_factor, "block": args.block or 128,
                           "batch": args.batch or 4}, "trials": [], "cached": None, "fixed": True}
        cfg = replace(cfg, pair_skin_factor=tuning["best"]["skin_factor"])
    solver_steps = args.steps * chunk
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=args.shift_every, host_state=host,
                           diag_ring=max(solver_steps + (max(args.warmup, 3) + 4) * chunk + 64, 256),
                           device=dev)
    if tuning is not None:
        eng.set_block(tuning["best"]["block"])
        eng.set_batch(tuning["best"]["batch"])
    nf, nw = eng.n_fluid, eng.n_wall
    eng.step(max(args.warmup, 3) * chunk)
    torch.cuda.synchronize(dev)
    rebuilds_before = eng.status()["rebuilds"]

    def barrier():
        if dist is not None:
            dist.barrier()

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize(dev)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(eng.stream)
    for _ in range(args.steps):
        eng.step(chunk)
    stop.record(eng.stream)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(start.elapsed_time(stop), dist, dev)
    status = eng.status()
    ms_step = ms / args.steps
    ms_solver = ms / solver_steps
    value = whole_job_rate(nf, solver_steps, world, ms / 1e3)
    # every solver step's kernels, plus the conditional rebuild body once per
    # list pass that rebuilt during the timed steps
    kernels_per_step, kernels_per_rebuild = eng.graph_kernels()
    rebuild_passes = status["rebuilds"] - rebuilds_before
    launches = kernels_per_step * solver_steps + kernels_per_rebuild * rebuild_passes
    entries_f, entries_w = eng.row_entries()

    stage = {}
    for _ in range(3):
        for k, v in eng.step_timed().items():
            stage.setdefault(k, []).append(v)
    stage = {k: statistics.median(v) for k, v in stage.items()}
    diag = eng.diagnostics(eng.steps_done - 1, 1).cpu()[0]
    eng.close()
    del eng
    torch.cuda.empty_cache()

    # roofline: the force pass against HBM, and the step against the binding
    # one of HBM and the FP32 pipe (both peaks measured here by the library's
    # probes unless the driver's HBM figure is present)
    probes = probe_peaks(dev)
    dp = driver_peaks()
    hbm_peak = float(dp["hbm_gbs"]) if dp and "hbm_gbs" in dp else probes["copy_gbs"]
    hbm_src = ("measured (MEASURED_PEAKS.json hbm_gbs)" if dp and "hbm_gbs" in dp
               else "measured in this run (tsph_probe_copy)")
    fp32_peak = probes["fp32_tflops"]
    t_force = stage["force"] / 1e3
    achieved = ALGO_BYTES_FORCE * nf / t_force / 1e9
    shift_passes = 1 if args.shift_every else 0
    flops_step = (entries_f * (PAIR_FLOPS["density"] + PAIR_FLOPS["diffusion"] + PAIR_FLOPS["force"]
                               + shift_passes * (PAIR_FLOPS["concentration"] + PAIR_FLOPS["gradient"]))
                  + entries_w * PAIR_FLOPS["walls"])
    bytes_step = ALGO_BYTES_STEP * nf + ALGO_BYTES_WALL * nw
    t_hbm = bytes_step / (hbm_peak * 1e9)
    t_fp32 = flops_step / (fp32_peak * 1e12)
    binding = {"bound": "fp32" if t_fp32 > t_hbm else "hbm",
               "frac": max(t_hbm, t_fp32) / (ms_solver / 1e3),
               "hbm_frac": t_hbm / (ms_solver / 1e3), "fp32_frac": t_fp32 / (ms_solver / 1e3),
               "bytes_per_step": bytes_step, "flops_per_step": flops_step,
               "fp32_tflops_achieved": flops_step / (ms_solver / 1e3) / 1e12,
               "row_entries": {"fluid": entries_f, "wall": entries_w},
               "flops_per_entry": PAIR_FLOPS,
               "note": "solver-step time against max(bytes / HBM peak, FLOPs / FP32 peak); FLOPs "
                       "counted from the kernel source per listed neighbour"}

    e2e = None
    if not args.no_e2e:
        x, m, w, n_ob = host
        pinned = tuple(t.pin_memory() for t in (x, m, w))
        from tensorsph_b200.engine import DIAG_FIELDS
        rows = torch.empty((args.steps, len(DIAG_FIELDS)), dtype=torch.float64).pin_memory()
        final = torch.empty((nf, 3), dtype=torch.float64).pin_memory()
        barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        e = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=args.shift_every,
                             host_state=(pinned[0], pinned[1], pinned[2], n_ob),
                             diag_ring=solver_steps + 8, device=dev)
        if tuning is not None:
            e.set_block(tuning["best"]["block"])
            e.set_batch(tuning["best"]["batch"])
        for k in range(args.steps):
            e.step(chunk)
            with torch.cuda.stream(e.stream):
                rows[k].copy_(e.diagnostics((k + 1) * chunk - 1, 1)[0], non_blocking=True)
        xs = e.state()[0]
        with torch.cuda.stream(e.stream):
            final.copy_(xs, non_blocking=True)
        torch.cuda.synchronize(dev)
        t_e2e = time.perf_counter() - t0
        barrier()
        t_e2e = max_over_ranks(t_e2e, dist, dev)
        e.close()
        state_bytes = (x.numel() + m.numel() + w.numel()) * 8
        e2e = {"value": whole_job_rate(nf, solver_steps, world, t_e2e), "unit": "fluid particle-updates/s",
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": rows.shape[1] * 8 + nf * 3 * 8 / args.steps,
               "scope": "engine creation from pinned host lattices + K bench steps with a meter-row "
                        "read each + final positions read, wall clock"}
        torch.cuda.empty_cache()

    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and args.cpu_sample_steps > 0:
        # the reference's own CPU code, and the FP64 oracle port with the
        # engine's field errors against it, on the 4x coarser rung
        port = None
        try:
            accuracy = oracle_port_and_errors(args.ref_dx, dev, args.shift_every, tuning)
            port = accuracy.pop("port")
        except Exception as exc:  # reported, never hides the headline
            accuracy = {"error": f"{type(exc).__name__}: {exc}"}
        if reference_available():
            r = reference_loop(args.ref_dx, args.ref_sample_steps, 1, args.shift_every)
            cpu = {"value": r["value"], "unit": "fluid particle-updates/s", "cores": r["cores"],
                   "kind": "reference",
                   "sample": f"{args.ref_sample_steps} solver steps after 1 warm-up step of the "
                             f"dx={args.ref_dx:g} rung ({r['fluid']} fluid): tensorsph from baseline/_ref, "
                             f"torch {r['torch']} {r['dtype']} on {r['cores']} threads ({r['cpu']}), "
                             f"{r['seconds']:.1f} s", "port": port}
        elif port is not None:
            cpu = dict(port)
        torch.cuda.empty_cache()

    extra = {}
    if rank == 0 and world == 1 and args.ckpt_steps > 0:
        try:
            extra["checkpoint"] = checkpoint_leg(args, dev, cfg, obstacle, host, tuning)
        except Exception as exc:  # reported, never hides the headline
            extra["checkpoint"] = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.empty_cache()
    if rank == 0 and world == 1:
        for name, leg, on in (("ensemble", ensemble_leg, args.ensemble_cases > 0),
                              ("serving", serving_leg, args.serve_requests > 0),
                              ("delta_plus_3d", delta_plus_leg, args.dplus_dx > 0),
                              ("shear", shear_leg, args.shear_steps > 0),
                              ("csf3", csf3_leg, args.csf3_radius > 0),
                              ("tvc", tvc_leg, args.tvc_n > 0),
                              ("rhs2d", rhs2d_leg, args.rhs2d_dx > 0)):
            if not on:
                continue
            try:
                extra[name] = leg(args, dev)
            except Exception as exc:  # reported, never hides the headline
                extra[name] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": "particle-updates/s", "value": value, "unit": "fluid particle-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded lattice, no dataset)",
            "config": {**workload_config(args), "fluid_particles": nf, "wall_particles": nw,
                       "solver_steps_per_step": chunk, "ms_per_solver_step": ms_solver,
                       "pair_skin_factor": cfg.pair_skin_factor,
                       "tuning": None if tuning is None else tuning["best"],
                       "pairs": "FP32 pair arithmetic, FP64 positions/velocities/meters",
                       "l2": "working set (state + neighbour rows) > 126 MB L2, no flush",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": binding["bound"], "kernel": "k_force", "achieved": achieved,
                         "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": FORCE_TRAFFIC_PER_FLUID * nf,
                         "traffic_source": f"from_profile: {FORCE_TRAFFIC_RUNG}",
                         "limiter": FORCE_LIMITER,
                         "peak_source": hbm_src,
                         "algorithmic_bytes_per_launch": ALGO_BYTES_FORCE * nf,
                         "launch_ms": stage["force"],
                         "step_hbm_frac": bytes_step / (ms_solver / 1e3) / 1e9 / hbm_peak,
                         "step_binding": binding},
            "peaks": {**probes, "hbm_gbs_used": hbm_peak,
                      "driver": dp if dp else "MEASURED_PEAKS.json absent"},
            "stage_ms": stage,
            "clocks": clocks,
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "errors_vs_fp64": accuracy,
            "engine": {"rebuilds": status["rebuilds"], "escapes": status["escapes"],
                       "obstacle_clamps": status["clamps"], "longest_row": status["row_max"],
                       "last_rho_max": float(diag[0]), "last_speed_max": float(diag[1]),
                       "kernels_per_step": kernels_per_step, "kernels_per_rebuild_pass": kernels_per_rebuild,
                       "rebuild_passes_timed": rebuild_passes},
        }
        line.update(extra)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
