"""3-D case lattices (``tensorsph.threed.solver`` set-up helpers)."""
from __future__ import annotations

import torch

__all__ = ["cubic_lattice", "wall_shell", "hydrostatic_density", "acoustic_dt", "COURANT"]

COURANT = 0.25


def acoustic_dt(dx: float, h: float, sound_speed: float, courant: float = COURANT) -> float:
    return courant * h / sound_speed


def cubic_lattice(shape, dx: float, origin=(0.0, 0.0, 0.0), dtype=torch.float64) -> torch.Tensor:
    """``shape = (nx, ny, nz)`` points, ``indexing='ij'`` order (x slowest)."""
    axes = [torch.arange(n, dtype=dtype) * dx + origin[axis] for axis, n in enumerate(shape)]
    grid = torch.meshgrid(*axes, indexing="ij")
    return torch.stack(grid, dim=-1).reshape(-1, len(shape))


def wall_shell(fluid_shape, layers: int, dx: float, dtype=torch.float64) -> torch.Tensor:
    """Lattice points of a ``layers``-thick shell around a ``fluid_shape`` block."""
    outer = tuple(int(n) + 2 * int(layers) for n in fluid_shape)
    axes = [torch.arange(n, dtype=dtype) * dx for n in outer]
    grid = torch.meshgrid(*axes, indexing="ij")
    index = torch.meshgrid(*[torch.arange(n) for n in outer], indexing="ij")
    inside = None
    for axis, n in enumerate(fluid_shape):
        m = (index[axis] >= layers) & (index[axis] < layers + int(n))
        inside = m if inside is None else inside & m
    return torch.stack(grid, dim=-1)[~inside]


def hydrostatic_density(z, height, rho0, sound_speed, gamma, gravity):
    stiffness = rho0 * sound_speed ** 2 / gamma
    p = rho0 * gravity * (height - z).clamp_min(0.0)
    return rho0 * (1.0 + p / stiffness) ** (1.0 / gamma)
