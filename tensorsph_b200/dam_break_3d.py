"""Drop-in 3-D dam-break pass on the B200 (``tensorsph.dam_break_3d``).

``rhs_3d`` keeps the reference signature and return order
(dam_break_3d.py:290-422) and runs the fused CUDA gather kernels of
``csrc/wcsph.cu`` with the 3-D cubic spline ``sigma = 1 / (pi h^3)``.  The
case-setup helpers build the same lattices as the reference (same
``arange`` / ``meshgrid`` construction, so the same particle order).
The time loop lives in :mod:`tensorsph_b200.engine`.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from functools import lru_cache
import math

import torch

from . import _lib
from .droplet_impact import Config, cell_centres, hydrostatic_density, symmetric_rows
from .neighbor_search import grid_pairs
from .integrate import clamp_box

__all__ = ["DamBreak3DConfig", "make_column_3d", "wall_lattice_3d", "rhs_3d",
           "apply_boundary_3d", "cubic_spline_kernel_3d", "cubic_spline_gradient_3d",
           "pair_kernels_3d", "front_position_3d", "mass_3d"]


def cubic_spline_kernel_3d(r: torch.Tensor, h: float) -> torch.Tensor:
    q = r / h
    first = 1.0 - 1.5 * q.square() + 0.75 * q.pow(3)
    second = 0.25 * (2.0 - q).clamp_min(0).pow(3)
    shape = torch.where(q < 1.0, first, torch.where(q < 2.0, second, 0.0))
    return (1.0 / (math.pi * h ** 3)) * shape.clamp_min(0.0)


def cubic_spline_gradient_3d(delta: torch.Tensor, h: float, eps: float = 1.0e-12) -> torch.Tensor:
    r = torch.linalg.vector_norm(delta, dim=-1)
    q = r / h
    dshape = torch.where(q < 1.0, -3.0 * q + 2.25 * q.square(),
                         torch.where(q < 2.0, -0.75 * (2.0 - q).square(), 0.0))
    scale = (1.0 / (math.pi * h ** 3)) * dshape / (h * r.clamp_min(eps))
    return delta * scale.unsqueeze(-1)


def pair_kernels_3d(delta: torch.Tensor, h: float, eps: float = 1.0e-12):
    r = torch.linalg.vector_norm(delta, dim=-1)
    return cubic_spline_kernel_3d(r, h), cubic_spline_gradient_3d(delta, h, eps)


@dataclass
class DamBreak3DConfig(Config):
    """3-D dam-break parameters (field names and defaults of dam_break_3d.py:103-143)."""

    dx: float = 0.02
    tank_height: float = 0.6
    tank_depth: float = 0.3
    column_width: float = 0.15
    column_depth: float = 0.15
    column_height: float = 0.3
    pool_width: float = 1.0
    pool_depth: float = 0.6
    dt: float = 5.0e-5
    steps: int = 4000
    output_every: int = 100
    device: str = "cpu"
    hydrostatic_init: bool = True
    tvc_every: int = 0
    tvc_alpha: float | None = None
    tvc_scope_tol: float | None = None
    tvc_max_shift: float | None = None

    def tank_top(self) -> float:
        return float(self.tank_height)

    def dt_from_courant(self) -> float:
        return self.max_courant * self.h_factor * self.dx / self.sound_speed


@lru_cache(maxsize=64)
def _lattice_sum_3d(dx: float, h: float) -> float:
    half = int(math.ceil(2.0 * h / dx)) + 1
    n = torch.arange(-half, half + 1, dtype=torch.float64) * dx
    grid = torch.cartesian_prod(n, n, n)
    r = torch.linalg.vector_norm(grid, dim=1)
    return float(cubic_spline_kernel_3d(r, h).sum() * dx ** 3)


def mass_3d(dx: float, h_factor: float, rho0: float, calibrated: bool) -> float:
    """Lattice mass shared by the 3-D fluid and the wall quadrature."""
    if calibrated:
        return rho0 * dx ** 3 / _lattice_sum_3d(float(dx), float(h_factor * dx))
    return rho0 * dx ** 3


def make_column_3d(cfg: DamBreak3DConfig, device, seed: int | None = None):
    dx = cfg.dx
    xs = cell_centres(cfg.column_width, dx, device)
    ys = cell_centres(cfg.column_height, dx, device)
    zs = cell_centres(cfg.column_depth, dx, device)
    gx, gy, gz = torch.meshgrid(xs, ys, zs, indexing="xy")
    positions = torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), dim=-1)
    if seed is not None:
        gen = torch.Generator(device=device).manual_seed(seed)
        noise = torch.randn(positions.shape, generator=gen, device=device) * dx * 1e-4
        positions = positions + noise
    unit = mass_3d(dx, cfg.h_factor, cfg.rho0, cfg.density_calibration)
    if cfg.hydrostatic_init:
        mass = hydrostatic_density(positions[:, 1], cfg, surface=cfg.column_height) * (unit / cfg.rho0)
    else:
        mass = torch.full((positions.shape[0],), unit, device=device)
    return positions, mass


def wall_lattice_3d(cfg: DamBreak3DConfig, device, top: float | None = None) -> torch.Tensor:
    """Wall particles on the bottom and the four sides, ``wall_layers`` deep."""
    if cfg.wall_layers < 1:
        raise ValueError("wall_layers must be positive")
    dx, layers = cfg.dx, cfg.wall_layers
    top = cfg.tank_top() if top is None else float(top)
    tw, td = cfg.pool_width, cfg.tank_depth
    parts = []

    def grid3(xs, ys, zs):
        gx, gy, gz = torch.meshgrid(xs, ys, zs, indexing="xy")
        return torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), dim=-1)

    span_x = torch.arange(-(layers - 0.5) * dx, tw + (layers - 0.5) * dx, dx, device=device)
    span_z = torch.arange(-(layers - 0.5) * dx, td + (layers - 0.5) * dx, dx, device=device)
    for layer in range(1, layers + 1):
        parts.append(grid3(span_x, torch.full((1,), dx * 0.5 - layer * dx, device=device), span_z))
    cols_y = torch.arange(dx * 0.5, top, dx, device=device)
    for layer in range(1, layers + 1):
        parts.append(grid3(torch.full((1,), dx * 0.5 - layer * dx, device=device), cols_y, span_z))
    for layer in range(1, layers + 1):
        parts.append(grid3(torch.full((1,), tw - dx * 0.5 + layer * dx, device=device), cols_y, span_z))
    span_xw = torch.arange(dx * 0.5, tw, dx, device=device)
    for layer in range(1, layers + 1):
        parts.append(grid3(span_xw, cols_y, torch.full((1,), dx * 0.5 - layer * dx, device=device)))
    for layer in range(1, layers + 1):
        parts.append(grid3(span_xw, cols_y, torch.full((1,), td - dx * 0.5 + layer * dx, device=device)))
    return torch.cat(parts, dim=0)


def rhs_3d(pos, vel, mass, cfg: DamBreak3DConfig, pairs=None, wall=None, dt=None, *,
           return_wall_force=False):
    """3-D density, pressure and acceleration on the GPU (dam_break_3d.py:290-422),
    with the free-surface pressure closure when configured; returns
    ``(rho, p, acc[, reaction])`` on ``pos``'s device."""
    n = pos.shape[0]
    nw = wall.shape[0] if wall is not None else 0
    h = cfg.h_factor * cfg.dx
    step_dt = dt if dt is not None else cfg.dt
    if cfg.density_diffusion > 0.0 and cfg.density_diffusion_form != "molteni":
        raise ValueError("density_diffusion_rate implements the 'molteni' form only; the "
                         f"configured form is {cfg.density_diffusion_form!r}")
    out_device = pos.device
    dev = _lib.cuda_device(pos)
    dtype = pos.dtype
    code = _lib.dtype_code(dtype)
    P = _lib.to_dev(pos.detach(), dev)
    V = _lib.to_dev(vel.detach(), dev, dtype)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    Wp = _lib.to_dev(wall.detach(), dev, dtype) if nw else None
    if pairs is None:
        all_pos = torch.cat((P, Wp), dim=0) if nw else P
        pairs_dev, _, _ = grid_pairs(all_pos, 2.0 * h, row_limit=n)
    else:
        pairs_dev = _lib.to_dev(pairs, dev)
    rowptr, entries = symmetric_rows(pairs_dev, n + nw)
    prm = _lib.WcsphParams()
    prm.dim, prm.dtype, prm.n_fluid, prm.n_wall = 3, code, n, nw
    prm.flags = _lib.RHS_WALL_SELF | (_lib.RHS_SPLIT if return_wall_force else 0)
    if cfg.surface_pressure_closure:
        # dam_break_3d.py:339-342: the 2-D closure over the fluid pairs
        prm.flags |= _lib.RHS_SURFACE_CLOSURE
        prm.surface_donors = 1 if cfg.surface_pressure_donors == "all" else 0
        prm.surface_layers = max(1, int(cfg.surface_pressure_layers))
        prm.surface_threshold = float(cfg.surface_pressure_threshold)
    prm.diffusion_form = 0
    prm.h, prm.sigma = h, 1.0 / (math.pi * h ** 3)
    prm.rho0, prm.sound_speed, prm.gamma = cfg.rho0, cfg.sound_speed, cfg.gamma
    prm.gravity, prm.viscosity, prm.wall_friction = cfg.gravity, cfg.viscosity, cfg.wall_friction
    prm.diffusion_scale = (2.0 * cfg.density_diffusion * cfg.sound_speed * cfg.h_factor * cfg.dx
                           if cfg.density_diffusion > 0.0 else 0.0)
    prm.dt = float(step_dt)
    prm.wall_mass = float(torch.tensor(mass_3d(cfg.dx, cfg.h_factor, cfg.rho0,
                                               cfg.density_calibration), dtype=dtype))
    rho = torch.empty(n, dtype=dtype, device=dev)
    pressure = torch.empty(n, dtype=dtype, device=dev)
    acc = torch.empty((n, 3), dtype=dtype, device=dev)
    reaction = torch.zeros((nw, 3), dtype=dtype, device=dev) if return_wall_force else None
    face = torch.zeros(nw, dtype=dtype, device=dev) if return_wall_force else None
    io = _lib.WcsphIO(P.data_ptr(), V.data_ptr(), M.data_ptr(), _lib.ptr(Wp), None, None, None,
                      None, rowptr.data_ptr(), entries.data_ptr(), rho.data_ptr(),
                      pressure.data_ptr(), acc.data_ptr(), _lib.ptr(reaction), _lib.ptr(face))
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_wcsph_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_wcsph_rhs(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                                _lib.stream(dev)), "tsph_wcsph_rhs")
    result = (rho.to(out_device), pressure.to(out_device), acc.to(out_device))
    if not return_wall_force:
        return result
    return (*result, reaction.to(out_device))


def apply_boundary_3d(pos, vel, cfg: DamBreak3DConfig, top: float | None = None) -> int:
    th = cfg.tank_top() if top is None else float(top)
    return clamp_box(pos, vel, (0.0, 0.0, 0.0), (cfg.pool_width, th, cfg.tank_depth),
                     0.25 * cfg.dx)


def front_position_3d(pos: torch.Tensor, cfg: DamBreak3DConfig) -> float:
    if pos.numel() == 0:
        return 0.0
    return float(pos[:, 0].max())
