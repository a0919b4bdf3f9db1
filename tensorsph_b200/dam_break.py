"""2-D dam-break case helpers (``tensorsph.dam_break``) for the B200 pass.

``DamBreakConfig`` keeps the reference fields and defaults (dam_break.py:45-121)
and ``make_column`` builds the same floored lattice with the hydrostatic mass
profile (dam_break.py:143-175).  The stepping loop of this case runs through
:func:`tensorsph_b200.engine.run_dam_break_2d`.
"""
from __future__ import annotations

from dataclasses import dataclass
import math

import torch

from .droplet_impact import Config, cell_centres, hydrostatic_density, lattice_mass_unit

__all__ = ["DamBreakConfig", "make_column", "front_position", "validate_case"]


@dataclass
class DamBreakConfig(Config):
    dx: float = 0.01
    tank_height: float = 0.75
    column_width: float = 0.2
    column_height: float = 0.4
    pool_width: float = 2.0
    pool_depth: float = 0.75
    dt: float = 1.0e-4
    steps: int = 6000
    output_every: int = 100
    device: str = "cpu"
    hydrostatic_init: bool = True
    shift_every: int = 0
    shift_strength: float = 1.0
    shift_limit: float = 0.25
    shift_v_ref: float | None = None
    tvc_every: int = 0
    tvc_alpha: float | None = None
    tvc_scope: str = "all"
    tvc_bulk_c: float = 0.95
    tvc_bulk_g: float = 0.02
    tvc_max_shift: float | None = None
    tvc_limiter: str | None = None
    tvc_limiter_slope: float = 100.0

    def tank_top(self) -> float:
        return float(self.tank_height)

    def dt_from_courant(self) -> float:
        return self.max_courant * self.h_factor * self.dx / self.sound_speed


def validate_case(cfg: DamBreakConfig) -> None:
    if cfg.boundary != "wall":
        raise ValueError("the dam-break case integrates static wall particles only; "
                         f"boundary={cfg.boundary!r} would be silently ignored")
    if cfg.dx <= 0 or cfg.h_factor <= 0:
        raise ValueError("dx and h_factor must be positive")
    if cfg.column_width <= 0 or cfg.column_height <= 0:
        raise ValueError("column dimensions must be positive")
    if cfg.column_width > cfg.pool_width or cfg.column_height > cfg.tank_height:
        raise ValueError("the column must fit inside the tank")
    if cfg.sound_speed <= 0 or cfg.rho0 <= 0 or cfg.gamma <= 0:
        raise ValueError("rho0, sound_speed, and gamma must be positive")
    courant = cfg.dt * cfg.sound_speed / (cfg.h_factor * cfg.dx)
    if courant > cfg.max_courant * (1.0 + 1.0e-9):
        raise ValueError(f"dt={cfg.dt:g} gives acoustic Courant {courant:.3f} > max_courant "
                         f"{cfg.max_courant:g}; use dt <= {cfg.dt_from_courant():.3e} s")


def make_column(cfg: DamBreakConfig, device):
    xs = cell_centres(cfg.column_width, cfg.dx, device)
    ys = cell_centres(cfg.column_height, cfg.dx, device)
    gx, gy = torch.meshgrid(xs, ys, indexing="xy")
    positions = torch.stack((gx.reshape(-1), gy.reshape(-1)), dim=-1)
    unit = lattice_mass_unit(cfg)
    if cfg.hydrostatic_init:
        mass = hydrostatic_density(positions[:, 1], cfg, surface=cfg.column_height) * (unit / cfg.rho0)
    else:
        mass = torch.full((positions.shape[0],), unit, device=device)
    return positions, mass


def front_position(pos: torch.Tensor, cfg: DamBreakConfig) -> float:
    if pos.numel() == 0:
        return 0.0
    return float(pos[:, 0].max())
