"""Drop-in 2-D WCSPH pair pass on the B200 (``tensorsph.droplet_impact``).

The public surface mirrors the reference module (droplet_impact.py): the
``Config`` dataclass with the same fields and defaults, the kernel helpers,
the EOS, the case-setup lattices and ``rhs`` with its full signature and
return contract.  ``rhs`` runs entirely in CUDA (``csrc/wcsph.cu``): the pair
list is turned into per-particle gather rows once, then four fused kernels
produce density (+ diffusion), the Adami wall state, and the acceleration.

The compression density regularisation and the free-surface pressure
closure run as two more kernels between the density and the wall pass; CSF
surface tension runs through the 2-D CSF drop-in over the fluid pairs.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from functools import lru_cache
import math

import torch

from . import _lib
from .neighbor_search import PairListCache, cell_linked_pairs, grid_pairs

__all__ = [
    "Config", "SimulationUnstableError", "VISCOUS_LAPLACIAN_FACTOR",
    "cubic_spline_kernel", "cubic_spline_gradient", "wendland_c2_kernel",
    "wendland_c2_gradient", "pair_kernels", "tait_pressure", "acoustic_courant",
    "suggested_dt", "viscous_dt_limit", "diffusion_dt_limit", "gravity_dt_limit",
    "validate_config", "hydrostatic_density", "lattice_kernel_sum",
    "calibrated_particle_mass", "lattice_mass_unit", "cell_centres", "pool_lattice",
    "make_particles", "wall_lattice", "wall_mass", "drop_wall_wall_pairs", "rhs",
    "symmetric_rows", "boundary_box", "apply_boundary", "domain_top",
    "PairListCache", "cell_linked_pairs", "density_from_neighbor_pairs", "rhs_all_pairs",
    "acoustic_dt_limit", "capillary_dt_limit", "stable_dt", "next_dt",
]

VISCOUS_LAPLACIAN_FACTOR = 2.0


class SimulationUnstableError(FloatingPointError):
    """Raised when a run violates one of its numerical acceptance criteria."""


@dataclass
class Config:
    """Case configuration; field names and defaults follow the reference
    ``Config`` (droplet_impact.py:55-269) so existing configurations load
    unchanged."""

    dx: float = 0.025
    h_factor: float = 1.3
    rho0: float = 1000.0
    sound_speed: float = 20.0
    gamma: float = 7.0
    gravity: float = 9.81
    viscosity: float = 0.01
    dt: float = 4.0e-4
    steps: int = 750
    output_every: int = 50
    pool_width: float = 1.0
    pool_depth: float = 0.35
    drop_radius: float = 0.10
    drop_center_y: float = 0.49
    device: str = "auto"
    boundary: str = "wall"
    wall_layers: int = 3
    max_courant: float = 0.3
    max_density_error: float = 0.05
    max_mach: float = 0.10
    fail_fast: bool = True
    pair_skin_factor: float = 0.25
    hydrostatic_init: bool = False
    calibrate_initial_mass: bool = False
    wall_friction: float = 0.0
    density_diffusion: float = 0.0
    density_diffusion_form: str = "molteni"
    density_diffusion_eigenvalue_floor: float = 0.1
    density_calibration: bool = True
    adaptive_dt: bool = False
    dt_growth: float = 1.1
    dt_safety: float = 0.9
    surface_tension_coefficient: float = 0.0
    contact_angle: float | None = None
    contact_angle_reach: float = 2.0
    contact_angle_model: str = "rotate"
    csf_scheme: str = "consistent"
    csf_delta_normalization: str = "legacy"
    csf_curvature: str = "fit_quadratic"
    surface_pressure_closure: bool = False
    surface_pressure_threshold: float = 0.99
    surface_pressure_donors: str = "interior"
    surface_pressure_layers: int = 2
    density_renormalization: bool = False
    boundary_consistent_density: bool = False
    density_regularization: str = "none"
    compression_regularization_rule: str = "free_surface"
    compression_normalization: str = "reference_mean"
    transport_velocity: str = "off"
    transport_velocity_strength: float = 1.0
    transport_velocity_v_ref: float | None = None


# --------------------------------------------------------------- kernels ---

def _shape(q):
    first = 1.0 - 1.5 * q.square() + 0.75 * q.pow(3)
    second = 0.25 * (2.0 - q).clamp_min(0).pow(3)
    return torch.where(q < 1.0, first, torch.where(q < 2.0, second, 0.0))


def _dshape(q):
    return torch.where(q < 1.0, -3.0 * q + 2.25 * q.square(),
                       torch.where(q < 2.0, -0.75 * (2.0 - q).square(), 0.0))


def cubic_spline_kernel(r: torch.Tensor, h: float) -> torch.Tensor:
    """2-D cubic spline ``W(r, h)`` with ``sigma = 10 / (7 pi h^2)``."""
    q = r / h
    return (10.0 / (7.0 * math.pi * h * h)) * _shape(q).clamp_min(0.0)


def cubic_spline_gradient(delta: torch.Tensor, h: float, eps: float = 1.0e-12) -> torch.Tensor:
    """``grad_i W`` for ``delta = x_i - x_j`` (2-D normalisation)."""
    r = torch.linalg.vector_norm(delta, dim=-1)
    scale = (10.0 / (7.0 * math.pi * h * h)) * _dshape(r / h) / (h * r.clamp_min(eps))
    return delta * scale.unsqueeze(-1)


def wendland_c2_kernel(r: torch.Tensor, h: float) -> torch.Tensor:
    """2-D Wendland C2 ``W(r, h)`` with ``sigma = 7 / (4 pi h^2)``."""
    q = r / h
    t = (1.0 - 0.5 * q).clamp_min(0.0)
    return (7.0 / (4.0 * math.pi * h * h)) * t.pow(4) * (2.0 * q + 1.0)


def wendland_c2_gradient(delta: torch.Tensor, h: float, eps: float = 1.0e-12) -> torch.Tensor:
    r = torch.linalg.vector_norm(delta, dim=-1)
    q = r / h
    t = (1.0 - 0.5 * q).clamp_min(0.0)
    scale = (7.0 / (4.0 * math.pi * h * h)) * (-5.0 * q * t.pow(3)) / (h * r.clamp_min(eps))
    return delta * scale.unsqueeze(-1)


def pair_kernels(delta: torch.Tensor, h: float, eps: float = 1.0e-12):
    """``(W, grad W)`` of a batch of separations (2-D normalisation)."""
    r = torch.linalg.vector_norm(delta, dim=-1)
    return cubic_spline_kernel(r, h), cubic_spline_gradient(delta, h, eps)


def tait_pressure(rho: torch.Tensor, cfg: Config) -> torch.Tensor:
    """Tait EOS with the 0.01 ratio floor and the ``p >= 0`` clamp."""
    bulk = cfg.rho0 * cfg.sound_speed ** 2 / cfg.gamma
    ratio = (rho / cfg.rho0).clamp_min(0.01)
    return (bulk * (ratio.pow(cfg.gamma) - 1.0)).clamp_min(0.0)


# ------------------------------------------------------------ time steps ---

def acoustic_courant(dt: float, cfg: Config, max_speed: float = 0.0) -> float:
    return dt * (cfg.sound_speed + max_speed) / (cfg.h_factor * cfg.dx)


def suggested_dt(cfg: Config, max_courant: float | None = None) -> float:
    limit = cfg.max_courant if max_courant is None else max_courant
    return limit * cfg.h_factor * cfg.dx / cfg.sound_speed


def viscous_dt_limit(cfg: Config, safety: float = 0.125) -> float:
    if cfg.viscosity <= 0.0:
        return float("inf")
    h = cfg.h_factor * cfg.dx
    return safety * h * h / cfg.viscosity


def acoustic_dt_limit(cfg: Config, max_speed: float = 0.0) -> float:
    """Largest step with dt (c0 + |v|) / h <= max_courant (droplet_impact.py:510-519)."""
    return (cfg.max_courant * cfg.h_factor * cfg.dx
            / (cfg.sound_speed + max(0.0, max_speed)))


def capillary_dt_limit(cfg: Config, safety: float = 0.25) -> float:
    """Capillary-wave step limit safety / sqrt(sigma k^3 / rho0) with k = 1/h
    (surface_tension.py:294-318, surface_tension_dispersion.py:755-778);
    infinite without surface tension."""
    if cfg.surface_tension_coefficient <= 0.0:
        return float("inf")
    h = cfg.h_factor * cfg.dx
    k = 1.0 / h
    return safety / math.sqrt(cfg.surface_tension_coefficient * k ** 3 / cfg.rho0)


def stable_dt(cfg: Config, max_speed: float = 0.0) -> float:
    """The smallest of the acoustic (for |v|), viscous, gravity, diffusion and
    capillary limits (droplet_impact.py:522-534)."""
    return min(acoustic_dt_limit(cfg, max_speed), viscous_dt_limit(cfg), gravity_dt_limit(cfg),
               diffusion_dt_limit(cfg), capillary_dt_limit(cfg))


def next_dt(cfg: Config, dt: float, max_speed: float = 0.0) -> float:
    """The next adaptive step: dt_safety times the stable step, grown by at
    most dt_growth, never above the configured dt (droplet_impact.py:537-556)."""
    target = cfg.dt_safety * stable_dt(cfg, max_speed)
    grown = dt * cfg.dt_growth if cfg.dt_growth >= 1.0 else target
    return min(target, grown, cfg.dt)


def diffusion_dt_limit(cfg: Config, safety: float = 0.125) -> float:
    if cfg.density_diffusion <= 0.0:
        return float("inf")
    return safety * cfg.h_factor * cfg.dx / (cfg.density_diffusion * cfg.sound_speed)


def gravity_dt_limit(cfg: Config, safety: float = 0.25) -> float:
    if cfg.gravity <= 0.0:
        return float("inf")
    return safety * math.sqrt(cfg.h_factor * cfg.dx / cfg.gravity)


def validate_config(cfg: Config) -> None:
    """Parameter checks of droplet_impact.py:1319-1386 (the subset the pass uses)."""
    if cfg.dx <= 0 or cfg.dt <= 0 or cfg.h_factor <= 0:
        raise ValueError("dx, dt, and h_factor must be positive")
    if cfg.rho0 <= 0 or cfg.sound_speed <= 0 or cfg.gamma <= 0:
        raise ValueError("rho0, sound_speed, and gamma must be positive")
    if cfg.pair_skin_factor < 0:
        raise ValueError("pair_skin_factor must be non-negative")
    if not 0.0 <= cfg.wall_friction <= 1.0:
        raise ValueError("wall_friction must be in [0, 1]")
    if cfg.density_diffusion < 0.0:
        raise ValueError("density_diffusion must be non-negative")
    if cfg.density_diffusion_form not in ("molteni", "antuono"):
        raise ValueError("density_diffusion_form must be one of ('molteni', 'antuono'), "
                         f"got {cfg.density_diffusion_form!r}")
    if not 0.0 <= cfg.density_diffusion_eigenvalue_floor < 1.0:
        raise ValueError("density_diffusion_eigenvalue_floor must be in [0, 1)")
    if not 0.0 < cfg.max_courant <= 1.0:
        raise ValueError("max_courant must be in (0, 1]")
    courant = acoustic_courant(cfg.dt, cfg)
    if courant > cfg.max_courant * (1.0 + 1.0e-9):
        raise ValueError(f"dt={cfg.dt:g} gives acoustic Courant {courant:.3f} > max_courant "
                         f"{cfg.max_courant:g}; use dt <= {suggested_dt(cfg):.3e} s")
    if cfg.dt > viscous_dt_limit(cfg) * (1.0 + 1.0e-9):
        raise ValueError(f"dt={cfg.dt:g} exceeds the viscous limit {viscous_dt_limit(cfg):.3e} s")
    if cfg.dt > gravity_dt_limit(cfg) * (1.0 + 1.0e-9):
        raise ValueError(f"dt={cfg.dt:g} exceeds the gravity limit {gravity_dt_limit(cfg):.3e} s")
    if cfg.dt > diffusion_dt_limit(cfg) * (1.0 + 1.0e-9):
        raise ValueError(f"dt={cfg.dt:g} exceeds the density-diffusion limit "
                         f"{diffusion_dt_limit(cfg):.3e} s")


# ----------------------------------------------------------------- setup ---

def domain_top(cfg: Config) -> float:
    return cfg.drop_center_y + cfg.drop_radius + 2.0 * cfg.dx


def hydrostatic_density(y: torch.Tensor, cfg: Config, surface: float | None = None) -> torch.Tensor:
    bulk = cfg.rho0 * cfg.sound_speed ** 2 / cfg.gamma
    top = cfg.pool_depth if surface is None else surface
    depth = (top - y).clamp_min(0.0)
    return cfg.rho0 * (1.0 + cfg.rho0 * cfg.gravity * depth / bulk).pow(1.0 / cfg.gamma)


@lru_cache(maxsize=256)
def _lattice_sum(h: float, dx: float) -> float:
    reach = int(math.ceil(2.0 * h / dx)) + 1
    offsets = torch.arange(-reach, reach + 1, dtype=torch.float64) * dx
    gx, gy = torch.meshgrid(offsets, offsets, indexing="xy")
    r = torch.sqrt(gx.square() + gy.square()).reshape(-1)
    return float(cubic_spline_kernel(r, h).sum())


def lattice_kernel_sum(h: float, dx: float) -> float:
    """``sum_j W(|x_j - x_i|)`` over a full square lattice, in float64."""
    if h <= 0.0 or dx <= 0.0:
        raise ValueError("h and dx must be positive")
    return _lattice_sum(float(h), float(dx))


def calibrated_particle_mass(cfg: Config, dx: float | None = None, h: float | None = None) -> float:
    step = cfg.dx if dx is None else float(dx)
    smoothing = cfg.h_factor * step if h is None else float(h)
    return float(cfg.rho0 / lattice_kernel_sum(smoothing, step))


def lattice_mass_unit(cfg: Config) -> float:
    if cfg.density_calibration:
        return calibrated_particle_mass(cfg)
    return cfg.rho0 * cfg.dx * cfg.dx


def cell_centres(extent: float, dx: float, device) -> torch.Tensor:
    """Cell centres of the lattice that fits inside ``[0, extent]`` (floored count)."""
    ratio = float(extent) / float(dx)
    count = int(math.floor(ratio + 1.0e-9))
    if count < 1:
        raise ValueError(f"dx={dx:g} is too coarse for an extent of {extent:g} "
                         f"(only {ratio:.3f} cells fit)")
    return (torch.arange(count, device=device, dtype=torch.get_default_dtype()) + 0.5) * dx


def pool_lattice(cfg: Config, device) -> torch.Tensor:
    xs = cell_centres(cfg.pool_width, cfg.dx, device)
    ys = cell_centres(cfg.pool_depth, cfg.dx, device)
    gx, gy = torch.meshgrid(xs, ys, indexing="xy")
    return torch.stack((gx.reshape(-1), gy.reshape(-1)), dim=-1)


def make_particles(cfg: Config, device):
    """Pool plus circular drop on a regular lattice; returns ``(positions, mass)``."""
    dx = cfg.dx
    if cfg.drop_center_y - cfg.drop_radius <= cfg.pool_depth:
        raise ValueError("drop must start above the pool surface")
    pool = pool_lattice(cfg, device)
    xs = cell_centres(cfg.pool_width, dx, device)
    drop_y = torch.arange(cfg.drop_center_y - cfg.drop_radius,
                          cfg.drop_center_y + cfg.drop_radius, dx, device=device)
    if drop_y.numel() == 0:
        raise ValueError("drop_radius is too small for the particle spacing")
    gx, gy = torch.meshgrid(xs, drop_y, indexing="xy")
    candidate = torch.stack((gx.reshape(-1), gy.reshape(-1)), dim=-1)
    center = torch.tensor([cfg.pool_width * 0.5, cfg.drop_center_y], device=device)
    drop = candidate[torch.linalg.vector_norm(candidate - center, dim=-1) <= cfg.drop_radius]
    if drop.shape[0] == 0:
        raise ValueError("drop discretization produced no particles")
    positions = torch.cat((pool, drop), dim=0)
    unit = lattice_mass_unit(cfg)
    mass = torch.full((positions.shape[0],), unit, device=device)
    if cfg.hydrostatic_init:
        pool_mass = hydrostatic_density(pool[:, 1], cfg) * (unit / cfg.rho0)
        mass = torch.cat((pool_mass, mass[pool.shape[0]:]), dim=0)
    if cfg.calibrate_initial_mass:
        raise NotImplementedError("calibrate_initial_mass belongs to tensorsph.initial_density")
    return positions, mass


def wall_lattice(cfg: Config, device, top: float | None = None) -> torch.Tensor:
    """Static dummy wall particles: ``wall_layers`` rows on the bottom and both sides,
    half a spacing outside the fluid box, extended around the corners."""
    if cfg.wall_layers < 1:
        raise ValueError("wall_layers must be positive")
    dx, layers = cfg.dx, cfg.wall_layers
    top = domain_top(cfg) if top is None else float(top)
    span_x = torch.arange(-(layers - 0.5) * dx, cfg.pool_width + (layers - 0.5) * dx, dx,
                          device=device)
    columns = torch.arange(dx * 0.5, top, dx, device=device)
    parts = []
    for layer in range(1, layers + 1):
        y = torch.full_like(span_x[:1], dx * 0.5 - layer * dx)
        gx, gy = torch.meshgrid(span_x, y, indexing="xy")
        parts.append(torch.stack((gx.reshape(-1), gy.reshape(-1)), dim=-1))
    for layer in range(1, layers + 1):
        for x in (dx * 0.5 - layer * dx, cfg.pool_width - dx * 0.5 + layer * dx):
            gx, gy = torch.meshgrid(torch.full_like(columns[:1], x), columns, indexing="xy")
            parts.append(torch.stack((gx.reshape(-1), gy.reshape(-1)), dim=-1))
    return torch.cat(parts, dim=0)


def wall_mass(cfg: Config, count: int, device) -> torch.Tensor:
    return torch.full((count,), lattice_mass_unit(cfg), device=device)


def drop_wall_wall_pairs(pairs: torch.Tensor, fluid_count: int) -> torch.Tensor:
    """Remove pairs whose two particles are both walls (index >= fluid_count)."""
    if pairs.numel() == 0:
        return pairs
    i, j = pairs.unbind(dim=1)
    usable = (i < fluid_count) | (j < fluid_count)
    if bool(usable.all()):
        return pairs
    return pairs[usable]


# ----------------------------------------------------------- gather rows ---

def density_from_neighbor_pairs(pos, mass, h: float, pairs=None):
    """Density summation over an unordered pair list with each particle's self
    term (droplet_impact.py:761-788), 2-D cubic normalisation as the reference
    uses in any dimension.  On the GPU it is the shift kernel's concentration
    sum with the masses as weights."""
    if pos.ndim != 2 or mass.ndim != 1 or mass.shape[0] != pos.shape[0]:
        raise ValueError("pos must be (N, D) and mass must be (N,)")
    if pos.device != mass.device:
        raise ValueError("pos and mass must be on the same device")
    if not pos.is_floating_point() or not mass.is_floating_point():
        raise TypeError("pos and mass must be floating-point tensors")
    if not math.isfinite(float(h)) or h <= 0:
        raise ValueError("h must be finite and positive")
    if pairs is not None:
        if pairs.ndim != 2 or pairs.shape[1] != 2 or pairs.dtype != torch.long:
            raise ValueError("pairs must be a long tensor with shape (pair_count, 2)")
        if pairs.device != pos.device:
            raise ValueError("pairs and pos must be on the same device")
    from .particle_shifting import concentration
    return concentration(pos, mass.to(pos.dtype), float(h), pairs=pairs)


def symmetric_rows(pairs: torch.Tensor, nrows: int):
    """Turn a ``(P, 2)`` pair list (CUDA) into row-sorted symmetric gather rows."""
    L = _lib.lib()
    dev = pairs.device
    pairs = pairs.contiguous()
    npairs = int(pairs.shape[0])
    rowptr = torch.empty(nrows + 1, dtype=torch.long, device=dev)
    entries = torch.empty(max(2 * npairs, 1), dtype=torch.int32, device=dev)
    ws = _lib.workspace(L.tsph_csr_workspace_bytes(npairs, nrows), dev)
    rc = L.tsph_csr_from_pairs(pairs.data_ptr(), npairs, nrows, rowptr.data_ptr(),
                               entries.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(dev))
    if rc == _lib.ERR_INDEX:
        raise ValueError("pair indices must lie in [0, particle_count)")
    _lib.check(rc, "tsph_csr_from_pairs")
    return rowptr, entries


def _wall_mass_value(cfg: Config) -> float:
    # The reference builds the wall masses with torch.full in the default dtype
    # and concatenates them with the fluid masses, so the value is rounded to
    # the default dtype first.
    return float(torch.tensor(lattice_mass_unit(cfg), dtype=torch.get_default_dtype()))


def rhs(pos, vel, mass, cfg: Config, pairs=None, wall=None, dt=None, wall_vel=None,
        wall_accel=None, state=None, split: bool = False, wrap_width: float | None = None,
        nu_field: torch.Tensor | None = None, density_offset: torch.Tensor | None = None,
        *, _self_donor: bool = False):
    """2-D WCSPH right-hand side on the GPU; returns ``(rho, pressure, acc)``
    (plus ``{"reaction", "face_pressure"}`` when ``split``), on ``pos``'s device.

    Contract and arithmetic of droplet_impact.py:810-1228.  With
    ``density_regularization="compression"`` the call reads the inverse
    reference compression from ``state["compression"]`` (a fresh
    ``CompressionRegularization`` when absent) and writes the new one there,
    the particle count to ``state["compression_counted"]``.
    ``_self_donor``: the free-surface closure's "all" donors include the
    receiver itself, as in the dense formulation (``rhs_all_pairs``).
    """
    h = cfg.h_factor * cfg.dx
    n = pos.shape[0]
    step_dt = cfg.dt if dt is None else float(dt)
    if pos.shape[1] != 2:
        raise ValueError(f"rhs implements 2-D smoothing only, got {pos.shape[1]} dimensions")
    if cfg.surface_tension_coefficient > 0.0 and cfg.csf_scheme != "consistent":
        raise NotImplementedError("the neighbour-count CSF scheme (csf_scheme='legacy') is not part of "
                                  "the B200 particle pass")
    if cfg.density_diffusion > 0.0 and cfg.density_diffusion_form not in ("molteni", "antuono"):
        raise ValueError(f"unknown density_diffusion_form {cfg.density_diffusion_form!r}; "
                         "expected one of ('molteni', 'antuono')")
    if wall is not None:
        if wall.ndim != 2 or wall.shape[1] != pos.shape[1]:
            raise ValueError("wall must be (W, D) with the same D as pos")
        if wall.device != pos.device or wall.dtype != pos.dtype:
            raise ValueError("wall must share pos device and dtype")
    nw = 0 if wall is None else int(wall.shape[0])
    if nu_field is not None:
        if not torch.is_tensor(nu_field) or nu_field.shape != (n,):
            raise ValueError(f"nu_field must be a tensor of shape ({n},)")
        if nu_field.device != pos.device or nu_field.dtype != pos.dtype:
            raise ValueError("nu_field must share pos device and dtype")
        if not bool(torch.isfinite(nu_field).all()):
            raise ValueError("nu_field must be finite")
        if bool((nu_field < 0).any()):
            raise ValueError("nu_field must be non-negative")
    if wrap_width is not None:
        width = float(wrap_width)
        if not math.isfinite(width) or width <= 0.0:
            raise ValueError("wrap_width must be a positive finite length")
    if wall_vel is not None and nw and (wall_vel.shape != (nw, 2) or wall_vel.dtype != pos.dtype):
        raise ValueError("wall_vel must be (wall_count, pos.shape[1])")
    if wall_accel is not None and nw and (wall_accel.shape != (nw, 2)
                                          or wall_accel.dtype != pos.dtype):
        raise ValueError("wall_accel must be (wall_count, pos.shape[1])")
    if cfg.boundary_consistent_density and cfg.density_regularization != "none":
        raise ValueError("boundary_consistent_density cannot be combined with "
                         "density_regularization != 'none'")

    out_device = pos.device
    dev = _lib.cuda_device(pos)
    dtype = pos.dtype
    code = _lib.dtype_code(dtype)
    P = _lib.to_dev(pos.detach(), dev)
    V = _lib.to_dev(vel.detach(), dev, dtype)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    Wp = _lib.to_dev(wall.detach(), dev) if nw else None

    if pairs is None:
        all_pos = torch.cat((P, Wp), dim=0) if nw else P
        pairs_dev, _, _ = grid_pairs(all_pos, 2.0 * h, row_limit=n)
    else:
        if pairs.ndim != 2 or pairs.shape[1] != 2 or pairs.dtype != torch.long:
            raise ValueError("pairs must be a long tensor with shape (pair_count, 2)")
        if pairs.device != pos.device:
            raise ValueError("pairs and pos must be on the same device")
        pairs_dev = _lib.to_dev(pairs, dev)
    empty = pairs_dev.shape[0] == 0
    if density_offset is not None and not empty:
        if density_offset.shape != (n,) or density_offset.device != pos.device:
            raise ValueError("density_offset must match the fluid particles")
        if density_offset.dtype != dtype:
            raise ValueError("density_offset must have the fluid dtype")
        if cfg.density_regularization != "none" or cfg.density_renormalization:
            raise ValueError("density_offset requires unnormalised summation density")
    compression = cfg.density_regularization != "none" and not empty
    if compression:
        # droplet_impact.py:982-1006
        from .compression_regularization import NORMALIZATIONS, RULES, CompressionRegularization
        if cfg.density_regularization != "compression":
            raise ValueError(f"unknown density_regularization {cfg.density_regularization!r};"
                             " expected 'none' or 'compression'")
        if cfg.density_renormalization:
            raise ValueError("density_regularization='compression' replaces the summation density; "
                             "combining it with density_renormalization would normalise an "
                             "already-normalised field")
        if cfg.compression_regularization_rule not in RULES:
            raise ValueError(f"unknown compression_regularization_rule "
                             f"{cfg.compression_regularization_rule!r}; expected one of {RULES}")
        if cfg.compression_normalization not in NORMALIZATIONS:
            raise ValueError(f"unknown compression_normalization {cfg.compression_normalization!r}; "
                             f"expected one of {NORMALIZATIONS}")
        if cfg.density_diffusion > 0.0:
            raise ValueError("density_regularization='compression' and density_diffusion are two "
                             "different ways of obtaining the density; pick one")
        regularizer = None if state is None else state.get("compression")
        if regularizer is None:
            regularizer = CompressionRegularization(rule=cfg.compression_regularization_rule,
                                                    normalization=cfg.compression_normalization)

    rowptr, entries = symmetric_rows(pairs_dev, n + nw)
    prm = _lib.WcsphParams()
    prm.dim, prm.dtype, prm.n_fluid, prm.n_wall = 2, code, n, nw
    flags = 0
    if not empty:
        if cfg.density_renormalization:
            flags |= _lib.RHS_RENORMALIZE
        if cfg.boundary_consistent_density and nw:
            flags |= _lib.RHS_BOUNDARY_DENSITY
        if split:
            flags |= _lib.RHS_SPLIT
        if wrap_width is not None:
            flags |= _lib.RHS_WRAP_X
        if compression:
            flags |= _lib.RHS_COMPRESSION
        if cfg.surface_pressure_closure:
            flags |= _lib.RHS_SURFACE_CLOSURE
    prm.flags = flags
    comp_out = None
    if compression:
        prm.compression_rule = 1 if cfg.compression_regularization_rule == "free_surface" else 0
        prm.compression_kref = (float(regularizer.inverse_reference_compression)
                                if cfg.compression_normalization == "reference_mean" else 1.0)
        comp_out = torch.empty(2, dtype=torch.float64, device=dev)
    literal = cfg.surface_pressure_donors == "all"
    prm.surface_donors = (2 if _self_donor else 1) if literal else 0
    prm.surface_layers = max(1, int(cfg.surface_pressure_layers))
    prm.surface_threshold = float(cfg.surface_pressure_threshold)
    prm.diffusion_form = 1 if cfg.density_diffusion_form == "antuono" else 0
    prm.h = h
    prm.sigma = 10.0 / (7.0 * math.pi * h * h)
    prm.rho0, prm.sound_speed, prm.gamma = cfg.rho0, cfg.sound_speed, cfg.gamma
    prm.gravity, prm.viscosity, prm.wall_friction = cfg.gravity, cfg.viscosity, cfg.wall_friction
    prm.diffusion_scale = (0.0 if empty or cfg.density_diffusion <= 0.0 else
                           2.0 * cfg.density_diffusion * cfg.sound_speed * cfg.h_factor * cfg.dx)
    prm.eigen_floor = cfg.density_diffusion_eigenvalue_floor
    prm.dt = step_dt
    prm.wall_mass = _wall_mass_value(cfg) if nw else 0.0
    prm.wrap_width = float(wrap_width) if wrap_width is not None else 0.0
    prm.lattice_sum = lattice_kernel_sum(h, cfg.dx) if cfg.density_renormalization else 0.0

    rho = torch.empty(n, dtype=dtype, device=dev)
    pressure = torch.empty(n, dtype=dtype, device=dev)
    acc = torch.empty((n, 2), dtype=dtype, device=dev)
    reaction = torch.zeros((nw, 2), dtype=dtype, device=dev) if split else None
    face = torch.zeros(nw, dtype=dtype, device=dev) if split else None
    keep = [_lib.to_dev(x, dev, dtype) if x is not None else None
            for x in (wall_vel if nw else None, wall_accel if nw else None, nu_field,
                      None if empty else density_offset)]
    io = _lib.WcsphIO(P.data_ptr(), V.data_ptr(), M.data_ptr(), _lib.ptr(Wp), _lib.ptr(keep[0]),
                      _lib.ptr(keep[1]), _lib.ptr(keep[2]), _lib.ptr(keep[3]), rowptr.data_ptr(),
                      entries.data_ptr(), rho.data_ptr(), pressure.data_ptr(), acc.data_ptr(),
                      _lib.ptr(reaction), _lib.ptr(face), _lib.ptr(comp_out))
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_wcsph_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_wcsph_rhs(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                                _lib.stream(dev)), "tsph_wcsph_rhs")
    if compression:
        # the reduce writes the scalar after this call consumed it
        written, counted = comp_out.tolist()
        regularizer.inverse_reference_compression = written
        if cfg.compression_regularization_rule == "free_stream":
            # compression_regularization.py:164-184: rhs passes no indicator;
            # the scalar is already written, the state entry is not
            raise ValueError("rule 'free_stream' needs an indicator array")
        if state is not None:
            state["compression"] = regularizer
            state["compression_counted"] = int(counted)
    if cfg.surface_tension_coefficient > 0.0 and not empty:
        # droplet_impact.py:1210-1222: the consistent CSF over the fluid pairs
        # of the step's list, with the configuration's options and the walls
        fluid_pairs = pairs_dev[(pairs_dev[:, 0] < n) & (pairs_dev[:, 1] < n)]
        if fluid_pairs.shape[0]:
            from .csf_consistent import surface_tension_acceleration
            a_st, _ = surface_tension_acceleration(
                P, rho, M, fluid_pairs, h, float(cfg.surface_tension_coefficient), rho0=cfg.rho0, wall=Wp,
                contact_angle=cfg.contact_angle, contact_angle_reach=cfg.contact_angle_reach,
                curvature_scheme=cfg.csf_curvature, delta_normalization=cfg.csf_delta_normalization,
                contact_angle_model=cfg.contact_angle_model)
            acc = acc + a_st
    result = (rho.to(out_device), pressure.to(out_device), acc.to(out_device))
    if split and not empty:
        return (*result, {"reaction": reaction.to(out_device),
                          "face_pressure": face.to(out_device)})
    return result


def rhs_all_pairs(pos, vel, mass, cfg: Config, dt=None):
    """The reference's dense formulation (droplet_impact.py:1232-1281): every
    fluid particle against every other, no walls; ``(rho, pressure, acc)`` on
    ``pos``'s device.

    The kernel vanishes beyond 2h, so this is the pair pass over every pair
    within 2h (the device all-pairs search) with the dense formulation's
    choices: the Molteni diffusion term whatever form is configured, no
    density renormalisation, boundary-consistent density, density
    regularisation or surface tension, and a free-surface closure whose pair
    set includes each particle with itself (droplet_impact.py:1255-1259)."""
    from dataclasses import replace
    from .neighbor_search import brute_force_pairs
    dense = replace(cfg, density_diffusion_form="molteni", density_renormalization=False,
                    boundary_consistent_density=False, density_regularization="none",
                    surface_tension_coefficient=0.0)
    pairs = brute_force_pairs(pos, 2.0 * cfg.h_factor * cfg.dx)
    return rhs(pos, vel, mass, dense, pairs=pairs.to(pos.device), dt=dt, _self_donor=True)


# -------------------------------------------------------------- boundary ---

def boundary_box(cfg: Config, top: float | None = None):
    height = domain_top(cfg) if top is None else float(top)
    if cfg.boundary == "wall":
        return 0.0, cfg.pool_width, 0.0, height
    margin = 0.5 * cfg.dx
    return margin, cfg.pool_width - margin, margin, height


def apply_boundary(pos, vel, cfg: Config, top: float | None = None) -> int:
    """Clamp into the box, zero the normal velocity of escapes (in place); returns
    the escape count (droplet_impact.py:1293-1312)."""
    from .integrate import clamp_box
    x0, x1, y0, y1 = boundary_box(cfg, top)
    return clamp_box(pos, vel, (x0, y0), (x1, y1), 0.25 * cfg.dx)
