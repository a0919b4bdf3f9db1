"""The 3-D dam break advanced by delta-plus steps (``delta_plus_step3``).

The reference drives its 2-D delta-plus step from the SPHERIC test 19 loop
(spheric19.py:101-175): h = 2 dx, four wall layers whose stations carry the
normal of their face, the exact barotropic hydrostatic start
rho = rho0 exp(g (H - y) / c0^2) with m = rho dx^D, a Verlet pair cache at
2h + 0.3 dx, and each step's position, velocity and density taken from the
step.  This module is that loop for the 3-D dam break of ``DamBreak3DConfig``
(with the box obstacle of the headline case, its stations' normals those of
their nearest face), on the device: the pair cache's rebuild is the device
cell search, the step is ``delta_plus_step3``'s kernels, and the step size is
fixed at ``max_courant`` h / c0 (<= 0.3 h / c0, the step's acoustic limit).

Reported per step: the front (max x of the fluid, dam_break_3d.py:459-463),
the force of the fluid on the obstacle (the sum of its stations' reactions)
and the largest density deviation |rho / rho0 - 1|.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import math
import time

import torch

from ..dam_break_3d import DamBreak3DConfig, wall_lattice_3d
from ..delta_plus import delta_plus_step3
from ..neighbor_search import PairListCache

__all__ = ["DeltaPlus3DRun", "delta_plus_case_3d", "run_delta_plus_3d"]


@dataclass
class DeltaPlus3DRun:
    steps: int
    dt: float
    n_fluid: int
    n_wall: int
    front: list = field(default_factory=list)
    obstacle_force: list = field(default_factory=list)
    density_deviation: list = field(default_factory=list)
    max_shift_over_dx: float = 0.0
    rebuilds: int = 0
    seconds: float = 0.0
    final_positions: torch.Tensor | None = None
    final_velocity: torch.Tensor | None = None
    final_density: torch.Tensor | None = None


def _station_normals(wall: torch.Tensor, cfg: DamBreak3DConfig, n_tank: int, obstacle) -> torch.Tensor:
    """Unit normals of the stations: the floor layers (y < 0) +y, the x side
    walls +x, the z side walls +z (the sign of a slip ghost's normal is
    immaterial, spheric19.py:117-120); an obstacle station takes the normal of
    its nearest face."""
    normal = torch.zeros_like(wall)
    tank = wall[:n_tank]
    floor = tank[:, 1] < 0
    xside = ~floor & ((tank[:, 0] < 0) | (tank[:, 0] > cfg.pool_width))
    zside = ~floor & ~xside
    normal[:n_tank, 1] = floor.to(wall.dtype)
    normal[:n_tank, 0] = xside.to(wall.dtype)
    normal[:n_tank, 2] = zside.to(wall.dtype)
    if obstacle is not None and wall.shape[0] > n_tank:
        ob = wall[n_tank:]
        lo = torch.tensor(obstacle[0], dtype=wall.dtype)
        hi = torch.tensor(obstacle[1], dtype=wall.dtype)
        # faces -x, +x, +y (top), -z, +z; the bottom face stands on the floor
        dist = torch.stack((ob[:, 0] - lo[0], hi[0] - ob[:, 0], hi[1] - ob[:, 1],
                            ob[:, 2] - lo[2], hi[2] - ob[:, 2]), dim=1)
        face = dist.argmin(dim=1)
        axis = torch.tensor([0, 0, 1, 2, 2])[face]
        normal[n_tank + torch.arange(ob.shape[0]), axis] = 1.0
    return normal


def delta_plus_case_3d(cfg: DamBreak3DConfig, obstacle=None, dtype=torch.float64):
    """Host state of the 3-D delta-plus dam break: fluid positions, density,
    mass, wall stations (tank, then obstacle) and their normals, the number of
    obstacle stations."""
    from dataclasses import replace
    from ..dam_break_3d import make_column_3d
    from ..engine import clamp_out_of_obstacle_host, obstacle_lattice_3d
    cfg = replace(cfg, h_factor=2.0, wall_layers=4)
    pos, _ = make_column_3d(cfg, "cpu")
    pos = pos.double()
    tank = wall_lattice_3d(cfg, "cpu", top=cfg.tank_top()).double()
    n_ob = 0
    wall = tank
    if obstacle is not None:
        ob = obstacle_lattice_3d(obstacle[0], obstacle[1], cfg.dx)
        clamp_out_of_obstacle_host(pos, obstacle[0], obstacle[1], 0.01 * cfg.dx)
        wall = torch.cat((tank, ob))
        n_ob = ob.shape[0]
    normal = _station_normals(wall, cfg, tank.shape[0], obstacle)
    height = cfg.column_height
    density = cfg.rho0 * torch.exp(cfg.gravity * (height - pos[:, 1]) / cfg.sound_speed ** 2)
    mass = density * cfg.dx ** 3
    return (pos.to(dtype), density.to(dtype), mass.to(dtype), wall.to(dtype), normal.to(dtype), n_ob)


def run_delta_plus_3d(cfg: DamBreak3DConfig, steps: int, *, obstacle=None, dtype=torch.float64,
                      device=None, skin: float = 0.3, host_state=None) -> DeltaPlus3DRun:
    """``steps`` delta-plus steps of the 3-D dam break on the device."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    pos, rho, mass, wall, normal, n_ob = host_state or delta_plus_case_3d(cfg, obstacle, dtype)
    pos, rho, mass, wall, normal = (t.to(dev, dtype).contiguous() for t in (pos, rho, mass, wall, normal))
    vel = torch.zeros_like(pos)
    wall_vel = torch.zeros_like(wall)
    dx = cfg.dx
    h = 2.0 * dx
    c0 = cfg.sound_speed
    dt = cfg.max_courant * h / c0
    vref = math.sqrt(2.0 * cfg.gravity * cfg.column_height)
    n, nw = pos.shape[0], wall.shape[0]
    cache = PairListCache(2.0 * h, skin * dx, fluid_count=n)
    run = DeltaPlus3DRun(steps=steps, dt=dt, n_fluid=n, n_wall=nw)
    shift_max = torch.zeros((), dtype=dtype, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(steps):
        pairs, _ = cache.get(torch.cat((pos, wall)))
        st = delta_plus_step3(pos, vel, rho, mass, dx=dx, sound_speed=c0, reference_speed=vref, dt=dt,
                              rho0=cfg.rho0, gravity=cfg.gravity, viscosity=cfg.viscosity,
                              wall=wall, wall_velocity=wall_vel, wall_normal=normal, pairs=pairs)
        run.front.append(pos[:, 0].max())
        run.obstacle_force.append(st.wall_reaction[nw - n_ob:].sum(0) if n_ob
                                  else torch.zeros(3, dtype=dtype, device=dev))
        run.density_deviation.append((st.density / cfg.rho0 - 1.0).abs().max())
        shift_max = torch.maximum(shift_max, st.shift.norm(dim=1).max() / dx)
        pos, vel, rho = st.position, st.velocity, st.density
    torch.cuda.synchronize(dev)
    run.seconds = time.perf_counter() - t0
    run.front = [float(v) for v in run.front]
    run.obstacle_force = [t.double().cpu() for t in run.obstacle_force]
    run.density_deviation = [float(v) for v in run.density_deviation]
    run.max_shift_over_dx = float(shift_max)
    run.rebuilds = cache.rebuilds
    run.final_positions, run.final_velocity, run.final_density = pos, vel, rho
    return run


def main(argv=None) -> None:
    """``python -m tensorsph_b200.threed.delta_plus3 --dx 0.0138 --steps 20``:
    the dam break with the obstacle advanced by delta-plus steps on the current
    GPU (two untimed steps first), one line of timing and state."""
    import argparse
    from ..engine import obstacle_case
    ap = argparse.ArgumentParser()
    ap.add_argument("--dx", type=float, default=0.0138)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--fp64", action="store_true")
    args = ap.parse_args(argv)
    dtype = torch.float64 if args.fp64 else torch.float32
    cfg, ob = obstacle_case(dx=args.dx)
    host = delta_plus_case_3d(cfg, ob, dtype)
    run_delta_plus_3d(cfg, 2, obstacle=ob, dtype=dtype, host_state=host)
    run = run_delta_plus_3d(cfg, args.steps, obstacle=ob, dtype=dtype, host_state=host)
    print(f"fluid {run.n_fluid} stations {run.n_wall} steps {run.steps} "
          f"ms/step {1e3 * run.seconds / run.steps:.3f} rebuilds {run.rebuilds} "
          f"max |rho/rho0 - 1| {max(run.density_deviation):.4g} front {run.front[-1]:.6f}")


if __name__ == "__main__":
    main()
