"""The wall-bounded 3-D hydrostatic column (``tensorsph.threed.run_hydrostatic``).

threed/solver.py:328-484 as a drop-in: the same arguments, ``HydrostaticResult``
and profile dictionary (build_pressure_profile, solver.py:487-625, with its
odd-even and binning diagnostics), computed on the device.  The column is an
``nx x ny x nz`` cubic lattice inside ``wall_layers`` of static wall lattice on
all six faces (``lid=False`` drops the layers at and above the surface), the
density starts on the analytic hydrostatic profile, the pair list is built
once at 2h (the reference never rebuilds it), and each step is kick-drift-kick
with the wall rows pinned, the right-hand side being ``accelerations`` (the
device's threed operators).  Pressure and density samples stay on the device
until the profile is reduced.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import math

import torch

from .conservation import diagnostics
from .kernel3 import calibrated_particle_mass
from .neighbors3 import box_pairs
from .operators3 import accelerations
from .solver import acoustic_dt, cubic_lattice, hydrostatic_density, wall_shell

__all__ = ["HydrostaticResult", "run_hydrostatic", "build_pressure_profile"]


@dataclass
class HydrostaticResult:
    """Outcome of one wall-bounded hydrostatic run (threed/solver.py:328-349)."""

    dx: float
    h: float
    sound_speed: float
    gravity: float
    height: float
    dt: float
    steps: int
    fluid_particles: int
    wall_particles: int
    times: list = field(default_factory=list)
    bottom_pressure: list = field(default_factory=list)
    centre_of_mass_z: list = field(default_factory=list)
    profile: dict = field(default_factory=dict)
    diagnostics: list = field(default_factory=list)

    @property
    def analytic_bottom_pressure(self) -> float:
        return self.profile.get("rho0", 1000.0) * self.gravity * self.height


def run_hydrostatic(*, nx: int = 10, ny: int = 10, nz: int = 8, dx: float = 0.01,
                    h_factor: float = 1.3, wall_layers: int = 2,
                    sound_speed: float = 20.0, rho0: float = 1000.0,
                    gamma: float = 7.0, gravity: float = 9.81,
                    viscosity: float = 0.02, t_end: float | None = None,
                    dt: float | None = None, steps: int | None = None,
                    sample_every: int = 5, settle_fraction: float = 0.4,
                    wall_model: str = "adami", lid: bool = True,
                    density_diffusion: float = 0.0,
                    density_diffusion_form: str = "antuono",
                    dtype=torch.float64, device=None) -> HydrostaticResult:
    """Integrate a wall-bounded 3-D column and compare ``p(z)`` with ``rho0 g (H - z)``."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    height = nz * dx
    walls = wall_layers * dx
    if dt is None:
        dt = acoustic_dt(dx, h_factor * dx, sound_speed)
    if t_end is None:
        t_end = 40.0 * height / sound_speed + 0.05
    if steps is None:
        steps = int(math.ceil(t_end / dt))
    h = h_factor * dx

    fluid = cubic_lattice((nx, ny, nz), dx, origin=(walls, walls, walls), dtype=dtype)
    n_fluid = fluid.shape[0]
    # the Lagrangian lattice row of every fluid particle (0 = bottom row)
    row_index = torch.unique(fluid[:, 2], sorted=True, return_inverse=True)[1]
    mass_fluid = torch.full((n_fluid,), calibrated_particle_mass(dx, h, rho0), dtype=dtype)
    wall = wall_shell((nx, ny, nz), wall_layers, dx, dtype=dtype)
    if not lid:
        wall = wall[wall[:, 2] <= walls + height + 1e-12]
    mass_wall = torch.full((wall.shape[0],), calibrated_particle_mass(dx, h, rho0), dtype=dtype)

    pos = torch.cat((fluid, wall)).to(dev)
    mass = torch.cat((mass_fluid, mass_wall)).to(dev)
    vel = torch.zeros_like(pos)
    rho0_field = hydrostatic_density(fluid[:, 2], walls + height, rho0, sound_speed, gamma, gravity)
    pairs = box_pairs(pos, 2.0 * h)
    g = torch.tensor([0.0, 0.0, -gravity], dtype=dtype)

    result = HydrostaticResult(dx=dx, h=h, sound_speed=sound_speed, gravity=gravity, height=height,
                               dt=dt, steps=steps, fluid_particles=n_fluid,
                               wall_particles=int(wall.shape[0]))
    result.density_diffusion = density_diffusion
    result.density_diffusion_form = density_diffusion_form

    def rhs(p, v):
        return accelerations(p, v, mass, h, pairs, rho0=rho0, sound_speed=sound_speed, gamma=gamma,
                             viscosity=viscosity, gravity=g, n_fluid=n_fluid, wall_model=wall_model,
                             density_diffusion=density_diffusion, dt=dt,
                             density_diffusion_form=density_diffusion_form)

    acc, rho, pressure = rhs(pos, vel)
    wall_pos = pos[n_fluid:].clone()
    times, bottoms, coms, buckets = [], [], [], []
    sample_start = int(steps * (1.0 - settle_fraction))
    for k in range(steps + 1):
        if k >= sample_start and k % sample_every == 0:
            times.append(k * dt)
            bottoms.append(pressure[:n_fluid].max())
            coms.append(pos[:n_fluid, 2].mean())
            buckets.append({"z": pos[:n_fluid, 2].clone(), "p": pressure[:n_fluid].clone(),
                            "rho": rho[:n_fluid].clone()})
        if k == steps:
            break
        # kick-drift-kick on the fluid; the wall rows stay pinned
        vel = vel + 0.5 * dt * acc
        vel[n_fluid:] = 0.0
        pos = pos + dt * vel
        pos[n_fluid:] = wall_pos
        acc, rho, pressure = rhs(pos, vel)
        vel = vel + 0.5 * dt * acc
        vel[n_fluid:] = 0.0
    wall_displacement = float((pos[n_fluid:] - wall_pos).abs().max()) if wall.shape[0] else 0.0

    result.times = times
    result.bottom_pressure = [float(b) for b in bottoms]
    result.centre_of_mass_z = [float(c) for c in coms]
    result.profile = build_pressure_profile(
        buckets, nz=nz, dx=dx, walls=walls, height=height, rho0=rho0, gravity=gravity, h=h,
        sound_speed=sound_speed, gamma=gamma, row_index=row_index.to(dev))
    result.profile["wall_model"] = wall_model
    result.profile["wall_displacement"] = wall_displacement
    result.diagnostics = [diagnostics(fluid.to(dev), vel[:n_fluid], mass[:n_fluid], rho0_field.to(dev),
                                      rho0=rho0, sound_speed=sound_speed, gamma=gamma)]
    return result


def _odd_even(values, scale: float):
    """Amplitude of the even/odd (checkerboard) mode of a layer sequence."""
    if len(values) < 4:
        return None
    even, odd = values[0::2], values[1::2]
    return abs(sum(even) / len(even) - sum(odd) / len(odd)) / scale


def _binning_diagnostic(z, layer, row_index, dx: float, walls: float):
    """How far the Eulerian layer bins are from one lattice row per bin."""
    if row_index is None or z.numel() == 0:
        return None
    samples = z.numel() // int(row_index.numel())
    label = torch.tile(row_index.to(torch.int64).reshape(-1), (samples,))
    offset = z - (walls + (layer.to(z.dtype) + 0.5) * dx)
    return {"mean_offset_over_dx": float(offset.mean()) / dx,
            "rms_offset_over_dx": float(torch.sqrt((offset * offset).mean())) / dx,
            "misplaced_fraction": float((layer != label).to(z.dtype).mean()),
            "rows": int(label.max()) + 1, "bins": int(layer.max()) + 1}


def build_pressure_profile(buckets, *, nz: int, dx: float, walls: float, height: float, rho0: float,
                           gravity: float, h: float, sound_speed: float, gamma: float,
                           row_index=None) -> dict:
    """Time-averaged p(z) over one-layer bins (Eulerian ``rows``, bins of
    floor((z - walls) / dx)) and over the particles' own lattice rows
    (``rows_by_lattice``), against rho0 g (H - z); accuracy numbers over the
    layers whose support is complete (3h below the surface), the depth
    integral and the odd-even amplitude (threed/solver.py:487-625)."""
    z = torch.cat([b["z"] for b in buckets])
    p = torch.cat([b["p"] for b in buckets])
    rho = torch.cat([b["rho"] for b in buckets])
    surface = walls + height
    layer = torch.clamp(((z - walls) / dx).floor().to(torch.int64), 0, nz - 1)
    count = torch.bincount(layer, minlength=nz)
    psum = torch.zeros(nz, dtype=p.dtype, device=p.device).index_add_(0, layer, p)
    rsum = torch.zeros(nz, dtype=rho.dtype, device=rho.device).index_add_(0, layer, rho)
    count_l, psum_l, rsum_l = count.tolist(), psum.tolist(), rsum.tolist()
    rows = []
    for index in range(nz):
        if count_l[index] == 0:
            continue
        z_centre = walls + (index + 0.5) * dx
        p_measured = psum_l[index] / count_l[index]
        p_analytic = rho0 * gravity * (surface - z_centre)
        rows.append({
            "layer": index, "z": z_centre, "depth_below_surface": surface - z_centre,
            "particles": count_l[index], "p_measured": p_measured, "p_analytic": p_analytic,
            "p_rel_error": (p_measured - p_analytic) / p_analytic if p_analytic > 0.0 else None,
            "rho_measured": rsum_l[index] / count_l[index],
            "rho_analytic": float(hydrostatic_density(torch.tensor(z_centre, dtype=torch.float64), surface,
                                                      rho0, sound_speed, gamma, gravity)),
            "support_complete": bool(z_centre < surface - 3.0 * h)})
    core = [r for r in rows if r["support_complete"]]
    scale = rho0 * gravity * height
    lattice_rows: list[dict] = []
    if row_index is not None and z.numel():
        samples = z.numel() // int(row_index.numel())
        label = torch.tile(row_index.to(torch.int64).reshape(-1), (samples,))
        nrow = int(label.max()) + 1
        cnt = torch.bincount(label, minlength=nrow).tolist()
        zs = torch.zeros(nrow, dtype=z.dtype, device=z.device).index_add_(0, label, z).tolist()
        ps = torch.zeros(nrow, dtype=p.dtype, device=p.device).index_add_(0, label, p).tolist()
        rs = torch.zeros(nrow, dtype=rho.dtype, device=rho.device).index_add_(0, label, rho).tolist()
        for index in range(nrow):
            if cnt[index] == 0:
                continue
            z_row = zs[index] / cnt[index]
            z_nominal = walls + index * dx
            p_measured = ps[index] / cnt[index]
            p_analytic = rho0 * gravity * (surface - z_row)
            lattice_rows.append({
                "row": index, "z": z_row, "z_nominal": z_nominal,
                "z_offset_over_dx": (z_row - z_nominal) / dx, "depth_below_surface": surface - z_row,
                "particles": cnt[index] // samples, "p_measured": p_measured, "p_analytic": p_analytic,
                "p_rel_error": (p_measured - p_analytic) / p_analytic if p_analytic > 0.0 else None,
                "rho_measured": rs[index] / cnt[index],
                "support_complete": bool(z_nominal < surface - 3.0 * h)})
        for r in lattice_rows:
            if r["p_rel_error"] is None:
                r["support_complete"] = False
    core_lattice = [r for r in lattice_rows if r["support_complete"] and r["p_rel_error"] is not None]
    errors = [r["p_rel_error"] for r in core]
    integral_measured = sum(r["p_measured"] for r in rows) * dx
    integral_analytic = sum(r["p_analytic"] for r in rows) * dx
    return {
        "rho0": rho0, "surface": surface, "rows": rows, "core_layers": len(core),
        "max_rel_error_core": max((abs(e) for e in errors), default=None),
        "mean_rel_error_core": (sum(errors) / len(errors)) if errors else None,
        "layers_within_15pct": sum(1 for e in errors if abs(e) < 0.15),
        "max_abs_error_over_scale": max((abs(r["p_measured"] - r["p_analytic"]) / scale for r in core),
                                        default=None),
        "integral_p_measured": integral_measured, "integral_p_analytic": integral_analytic,
        "integral_rel_error": ((integral_measured - integral_analytic) / integral_analytic
                               if integral_analytic else None),
        "odd_even_amplitude_over_scale": _odd_even([r["p_measured"] for r in rows], scale),
        "bottom_pressure_measured": rows[0]["p_measured"] if rows else None,
        "bottom_pressure_analytic": rows[0]["p_analytic"] if rows else None,
        "binning": _binning_diagnostic(z, layer, row_index, dx, walls),
        "rows_by_lattice": lattice_rows, "core_layers_lattice": len(core_lattice),
        "max_rel_error_core_lattice": max((abs(r["p_rel_error"]) for r in core_lattice), default=None),
        "mean_rel_error_core_lattice": (sum(r["p_rel_error"] for r in core_lattice) / len(core_lattice)
                                        if core_lattice else None),
        "layers_within_15pct_lattice": sum(1 for r in core_lattice if abs(r["p_rel_error"]) < 0.15),
        "max_abs_error_over_scale_lattice": max((abs(r["p_measured"] - r["p_analytic"]) / scale
                                                 for r in core_lattice), default=None),
        "odd_even_amplitude_over_scale_lattice": _odd_even([r["p_measured"] for r in lattice_rows], scale),
    }
