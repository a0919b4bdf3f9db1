"""Device-resident multi-case engine (``csrc/engine.cu``) and its case drivers.

``BatchEngine`` owns a fixed block of HBM (its capacities) in which any number
of independent cases live at once: each case keeps FP64 positions, velocities
and meters, cell-sorted particles and a skin-cached neighbour list on the
device, and one CUDA graph advances every case by one step (skin test and
rebuild, density, Molteni diffusion, Tait, Adami walls, force, obstacle
reaction, semi-implicit Euler with the box and obstacle clamps).  Cases are
admitted and retired while the others keep running; a case evolves bit for
bit the same alone or in a batch.

``CaseSpec`` is one case ready for admission; ``dam_break_3d_case`` and
``dam_break_2d_case`` build it from the reference configurations.

``DamBreak3DEngine`` is the single-case engine (with the optional Lind shift)
and ``run_case`` / ``run_dam_break_2d`` are the drop-ins for
``tensorsph.dam_break_3d.run_case`` (dam_break_3d.py:569-734) and
``tensorsph.dam_break.run_case`` (dam_break.py:319-460).  ``obstacle_case``
builds the 3-D dam break with a box obstacle (fluid 1.2 x 1.0 x 0.55 m in a
3.2 x 1.0 x 1.0 m tank, obstacle 0.16 x 0.16 x 0.4 m).
"""
from __future__ import annotations

import ctypes
import functools
from dataclasses import dataclass, field
import math

import torch

from . import _lib
from .dam_break_3d import DamBreak3DConfig, make_column_3d, mass_3d, wall_lattice_3d

__all__ = ["BatchEngine", "CaseSpec", "DamBreak3DEngine", "DamBreak3DRun", "dam_break_2d_case",
           "dam_break_3d_case", "droplet_impact_case", "engine_bytes", "shear_decay_case", "obstacle_case", "obstacle_lattice_3d",
           "run_case", "run_dam_break_2d", "tune_single_case", "DIAG_FIELDS"]

MAX_ROWS = (1 << 26) - 2   # fluid + wall rows the host layer gives one engine (the engine takes < 2^31 - 1)
FIT_NEIGHBORS = 128        # CSF curvature-fit row capacity (2-D, 4h + skin)

DIAG_FIELDS = ("rho_max", "speed_max", "front", "force_x", "force_y", "force_z", "kinetic",
               "potential", "escapes", "clamps", "rebuilds", "row_max", "step", "status",
               "impulse_x", "c_reference", "tvc_max_shift", "tvc_shift_sum", "tvc_kept",
               "tvc_clipped", "impulse_y", "impulse_z", "clamp_impulse_x", "clamp_impulse_y",
               "clamp_impulse_z", "time", "dt", "dt_unclamped", "compression_inverse",
               "compression_counted")


def obstacle_lattice_3d(lo, hi, dx: float) -> torch.Tensor:
    """Solid particles filling the box ``[lo, hi]`` on the fluid lattice
    (kleefsman_obstacle_3d.py:187-205)."""
    def span(a, b):
        n = max(1, int(round((b - a) / dx)))
        return a + (torch.arange(n, dtype=torch.float64) + 0.5) * dx
    gx, gy, gz = torch.meshgrid(span(lo[0], hi[0]), span(lo[1], hi[1]), span(lo[2], hi[2]),
                                indexing="xy")
    return torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), dim=-1)


def clamp_out_of_obstacle_host(pos: torch.Tensor, lo, hi, eps: float) -> int:
    """Move fluid particles that start inside the obstacle out through the
    nearest face (set-up only, kleefsman_obstacle_3d.py:208-266)."""
    inside = torch.ones(pos.shape[0], dtype=torch.bool)
    for k in range(3):
        inside &= (pos[:, k] > lo[k]) & (pos[:, k] < hi[k])
    idx = inside.nonzero().reshape(-1)
    if idx.numel() == 0:
        return 0
    px = pos[idx]
    cand = torch.stack((px[:, 0] - lo[0], hi[0] - px[:, 0], px[:, 1] - lo[1], hi[1] - px[:, 1],
                        px[:, 2] - lo[2], hi[2] - px[:, 2]), dim=1)
    which = cand.argmin(dim=1)
    for f in range(6):
        k = f // 2
        sel = which == f
        px[sel, k] = (hi[k] + eps) if f % 2 else (lo[k] - eps)
    pos[idx] = px
    return int(idx.numel())


def obstacle_case(dx: float = 0.0069, *, viscosity: float = 1.0e-6, density_diffusion: float = 0.1,
                  steps: int = 5000, courant: float = 0.25):
    """Configuration and obstacle box of the 3-D dam break with an obstacle.

    Fluid block 1.2 x 1.0 x 0.55 m in a 3.2 x 1.0 x 1.0 m tank, three wall
    layers, Tait rho0 = 1000, gamma = 7, c0 = 10 sqrt(2 g 0.55), h = 1.3 dx,
    Molteni diffusion delta = 0.1, acoustic CFL 0.25.  The obstacle
    (0.16 streamwise x 0.16 high x 0.4 spanwise) stands on the floor, centred
    across the tank, its centre 0.744 m from the downstream wall.
    """
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 0.55)
    h = 1.3 * dx
    cfg = DamBreak3DConfig(dx=dx, pool_width=3.2, tank_depth=1.0, tank_height=1.0,
                           column_width=1.2, column_depth=1.0, column_height=0.55, wall_layers=3,
                           density_diffusion=density_diffusion, sound_speed=c0,
                           viscosity=viscosity, dt=courant * h / c0, max_courant=courant,
                           steps=steps)
    x0 = 3.2 - 0.744 - 0.08
    lo = (x0, 0.0, 0.3)
    hi = (x0 + 0.16, 0.16, 0.7)
    return cfg, (lo, hi)


# ------------------------------------------------------------------ cases --

@dataclass
class CaseSpec:
    """One case ready for admission: parameters plus its host arrays (FP64).

    ``wall`` holds the static wall particles with the obstacle particles, if
    any, as its last ``n_obstacle`` rows (the order of the reference's
    ``torch.cat((wall, obstacle))``); ``v`` None is a case at rest (its zero
    velocities are written on the device at admission)."""

    params: _lib.CaseParams
    x: torch.Tensor
    v: torch.Tensor | None
    mass: torch.Tensor
    wall: torch.Tensor
    label: str = ""

    @property
    def dim(self) -> int:
        return int(self.params.dim)

    @property
    def n_fluid(self) -> int:
        return int(self.params.n_fluid)

    @property
    def n_wall(self) -> int:
        return int(self.params.n_wall)

    @property
    def n_obstacle(self) -> int:
        return int(self.params.n_obstacle)

    @property
    def dt(self) -> float:
        return float(self.params.dt)

    def cells(self) -> int:
        n = _lib.lib().tsph_engine_case_cells(ctypes.byref(self.params))
        if n < 0:
            raise ValueError("invalid case parameters")
        return int(n)


def _case_params(*, dim, n_fluid, n_wall, n_obstacle, cfg, h, wall_mass, box_hi, lo, hi,
                 shift_every=0, obstacle=None, first_step=0, adaptive=False, start_clock=None):
    psi = cfg.density_diffusion > 0.0 and cfg.density_diffusion_form == "antuono"
    if psi and dim == 3:
        # rhs_3d's contract (dam_break_3d.py:330-336)
        raise ValueError("density_diffusion_rate implements the 'molteni' form only; the "
                         f"configured form is {cfg.density_diffusion_form!r}")
    if dim == 3 and (cfg.density_renormalization or cfg.boundary_consistent_density):
        raise NotImplementedError("density_renormalization and boundary_consistent_density are "
                                  "options of the 2-D rhs")
    reg = getattr(cfg, "density_regularization", "none")
    compression = dim == 2 and reg != "none"
    if compression:
        # the rhs's contract (droplet_impact.py:982-1006); rhs_3d has no regularisation
        from .compression_regularization import NORMALIZATIONS, RULES
        if reg != "compression":
            raise ValueError(f"unknown density_regularization {reg!r}; expected 'none' or 'compression'")
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
        if cfg.compression_regularization_rule == "free_stream":
            # compression_regularization.py:164-184: the loop passes no indicator
            raise ValueError("rule 'free_stream' needs an indicator array")
        if cfg.boundary_consistent_density:
            raise ValueError("boundary_consistent_density cannot be combined with "
                             "density_regularization != 'none'")
    p = _lib.CaseParams()
    p.dim, p.n_fluid, p.n_wall, p.n_obstacle = dim, n_fluid, n_wall, n_obstacle
    p.shift_every = int(shift_every)
    p.first_step = int(first_step)
    p.has_obstacle = 1 if obstacle is not None else 0
    p.h, p.rho0, p.sound_speed, p.gamma = h, cfg.rho0, cfg.sound_speed, cfg.gamma
    p.gravity, p.viscosity, p.wall_friction = cfg.gravity, cfg.viscosity, cfg.wall_friction
    p.diffusion_scale = (2.0 * cfg.density_diffusion * cfg.sound_speed * cfg.h_factor * cfg.dx
                         if cfg.density_diffusion > 0.0 else 0.0)
    p.dt = cfg.dt
    p.wall_mass = wall_mass
    p.skin = cfg.pair_skin_factor * h
    # the psi diffusion form (density_diffusion.py:95-172) and the 2-D rhs's
    # density options (droplet_impact.py:954-964, 1090-1112)
    p.diffusion_form = 1 if psi else 0
    p.diffusion_eigen_floor = float(cfg.density_diffusion_eigenvalue_floor)
    if cfg.density_renormalization:
        from .droplet_impact import lattice_kernel_sum
        p.density_renormalization = 1
        p.lattice_kernel_sum = float(lattice_kernel_sum(h, cfg.dx))
    p.boundary_consistent_density = 1 if cfg.boundary_consistent_density else 0
    if compression:
        p.compression = 1
        p.compression_rule = 1 if cfg.compression_regularization_rule == "free_surface" else 0
        p.compression_normalization = 1 if cfg.compression_normalization == "reference_mean" else 0
    if getattr(cfg, "surface_pressure_closure", False):
        # droplet_impact.py:429-492 (rhs) and dam_break_3d.py:339-342 (rhs_3d)
        p.surface_closure = 1
        p.surface_threshold = float(cfg.surface_pressure_threshold)
        p.surface_donors = 1 if cfg.surface_pressure_donors == "all" else 0
        p.surface_layers = max(1, int(cfg.surface_pressure_layers))
    for k in range(3):
        p.box_hi[k] = box_hi[k]
    p.tolerance = 0.25 * cfg.dx
    if obstacle is not None:
        for k in range(3):
            p.ob_lo[k], p.ob_hi[k] = obstacle[0][k], obstacle[1][k]
        p.ob_eps = 0.01 * cfg.dx
    p.tvc_every = int(getattr(cfg, "tvc_every", 0) or 0)
    p.tvc_alpha, p.tvc_scope_tol, p.tvc_max_shift = 0.0, -1.0, -1.0
    p.tvc_slope, p.tvc_wall_volume, p.tvc_bulk_c = -1.0, -1.0, 0.0
    if p.tvc_every and (obstacle is not None or shift_every):
        raise NotImplementedError("the device engine runs the transport-velocity correction in the "
                                  "dam breaks without an obstacle or shifting")
    if p.tvc_every:
        # the module default 0.2 / 4 unless set; the clip is given in units of h
        p.tvc_alpha = 0.05 if cfg.tvc_alpha is None else float(cfg.tvc_alpha)
        p.tvc_max_shift = -1.0 if cfg.tvc_max_shift is None else float(cfg.tvc_max_shift) * h
        if dim == 3:
            # dam_break_3d.py:675-704: scope by |g| h, walls at m_w / rho0
            p.tvc_scope_tol = -1.0 if cfg.tvc_scope_tol is None else float(cfg.tvc_scope_tol)
        else:
            # dam_break.py:434-459: scope "all", "bulk_g" (|g| h <= tvc_bulk_g)
            # or "bulk" (C >= tvc_bulk_c c_ref after the update), the named
            # limiter, walls at dx^2
            scope = getattr(cfg, "tvc_scope", "all")
            if scope not in ("all", "bulk_g", "bulk"):
                raise ValueError(f"unknown tvc_scope {scope!r}")
            p.tvc_scope_tol = float(cfg.tvc_bulk_g) if scope == "bulk_g" else -1.0
            if scope == "bulk":
                if not cfg.tvc_bulk_c > 0.0:
                    raise ValueError("tvc_scope='bulk' needs tvc_bulk_c > 0")
                p.tvc_bulk_c = float(cfg.tvc_bulk_c)
            limiter = getattr(cfg, "tvc_limiter", None)
            if limiter == "truncated_linear":
                p.tvc_slope = float(cfg.tvc_limiter_slope)
            elif limiter not in (None, "none"):
                raise ValueError(f"unknown tvc_limiter {limiter!r}")
            p.tvc_wall_volume = float(cfg.dx) ** 2
    if adaptive:
        # next_dt (droplet_impact.py:522-556) on the device: the acoustic limit
        # there, the others are constants of the case
        from .droplet_impact import capillary_dt_limit, diffusion_dt_limit, gravity_dt_limit, viscous_dt_limit
        p.adaptive_dt = 1
        p.courant_h = cfg.max_courant * cfg.h_factor * cfg.dx
        p.dt_limit = min(viscous_dt_limit(cfg), gravity_dt_limit(cfg), diffusion_dt_limit(cfg),
                         capillary_dt_limit(cfg))
        p.dt_growth, p.dt_safety = float(cfg.dt_growth), float(cfg.dt_safety)
        p.target_time = cfg.steps * cfg.dt
        if start_clock is not None:
            # a resumed run: the time at the start of first_step and its step size
            p.start_elapsed, p.start_dt = float(start_clock[0]), float(start_clock[1])
    p.shift_strength = getattr(cfg, "shift_strength", 1.0)
    p.shift_limit = getattr(cfg, "shift_limit", 0.25)
    p.shift_free_surface = 0.95
    p.shift_vref_floor = 0.05 * cfg.sound_speed
    if getattr(cfg, "shift_v_ref", None) is not None:
        p.shift_vref_given, p.shift_vref = 1, float(cfg.shift_v_ref)
    margin = 2.0 * cfg.dx
    for k in range(3):
        if k < dim:
            p.grid_lo[k] = min(lo[k], 0.0) - margin
            p.grid_hi[k] = max(hi[k], box_hi[k]) + margin
    return p


def dam_break_3d_host_state(cfg: DamBreak3DConfig, obstacle=None, seed=None):
    """Host lattices of a 3-D case: fluid (FP64), masses, walls (+ obstacle
    particles last) and the obstacle particle count."""
    saved = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        x, mass = make_column_3d(cfg, "cpu", seed=seed)
        wall = wall_lattice_3d(cfg, "cpu")
        n_ob = 0
        if obstacle is not None:
            ob = obstacle_lattice_3d(obstacle[0], obstacle[1], cfg.dx)
            n_ob = ob.shape[0]
            wall = torch.cat((wall, ob))
            clamp_out_of_obstacle_host(x, obstacle[0], obstacle[1], 0.01 * cfg.dx)
    finally:
        torch.set_default_dtype(saved)
    return x.double(), mass.double(), wall.double(), n_ob


def dam_break_3d_case(cfg: DamBreak3DConfig, *, obstacle=None, shift_every: int = 0, seed=None,
                      host_state=None, velocity=None, first_step: int = 0, start_clock=None,
                      label: str = "") -> CaseSpec:
    """The 3-D dam break of ``tensorsph.dam_break_3d`` (optionally with the box
    obstacle of kleefsman_obstacle_3d.py) as a ``CaseSpec``; ``first_step``
    numbers the first step of a resumed run, and an adaptive run resumed from a
    checkpoint starts from ``start_clock`` = (elapsed, dt) of that checkpoint."""
    if host_state is None:
        host_state = dam_break_3d_host_state(cfg, obstacle, seed)
    x, mass, wall, n_ob = host_state
    x = x.double().contiguous()
    wall = wall.double().contiguous()
    h = cfg.h_factor * cfg.dx
    box = (cfg.pool_width, cfg.tank_top(), cfg.tank_depth)
    lo, hi = torch.aminmax(x, dim=0)
    if wall.shape[0]:
        wlo, whi = torch.aminmax(wall, dim=0)
        lo, hi = torch.minimum(lo, wlo), torch.maximum(hi, whi)
    p = _case_params(dim=3, n_fluid=x.shape[0], n_wall=wall.shape[0], n_obstacle=n_ob, cfg=cfg, h=h,
                     wall_mass=mass_3d(cfg.dx, cfg.h_factor, cfg.rho0, cfg.density_calibration),
                     box_hi=box, lo=lo.tolist(), hi=hi.tolist(), shift_every=shift_every,
                     obstacle=obstacle, first_step=first_step, adaptive=cfg.adaptive_dt,
                     start_clock=start_clock)
    v = None if velocity is None else velocity.double().contiguous()
    return CaseSpec(p, x, v, mass.double().contiguous(), wall, label or "dam_break_3d")


def dam_break_2d_case(cfg, *, shift_every: int = 0, velocity=None, label: str = "") -> CaseSpec:
    """The 2-D dam break of ``tensorsph.dam_break`` (dam_break.py:319-340 set-up:
    ``make_column`` and ``wall_lattice`` up to ``tank_top``) as a ``CaseSpec``."""
    from .dam_break import make_column, validate_case
    from .droplet_impact import lattice_mass_unit, wall_lattice
    validate_case(cfg)
    if cfg.surface_tension_coefficient > 0.0:
        raise NotImplementedError("surface tension in the dam-break case is not part of the device engine")
    x, mass = make_column(cfg, "cpu")
    wall = wall_lattice(cfg, "cpu", top=cfg.tank_top())
    x = x.double().contiguous()
    wall = wall.double().contiguous()
    h = cfg.h_factor * cfg.dx
    box = (cfg.pool_width, cfg.tank_top(), 0.0)
    allpos = torch.cat((x, wall))
    p = _case_params(dim=2, n_fluid=x.shape[0], n_wall=wall.shape[0], n_obstacle=0, cfg=cfg, h=h,
                     wall_mass=lattice_mass_unit(cfg), box_hi=box,
                     lo=allpos.min(dim=0).values.tolist(), hi=allpos.max(dim=0).values.tolist(),
                     shift_every=shift_every, adaptive=cfg.adaptive_dt)
    v = torch.zeros_like(x) if velocity is None else velocity.double().contiguous()
    return CaseSpec(p, x, v, mass.double().contiguous(), wall, label or "dam_break_2d")


def _wall_spacing(wall: torch.Tensor) -> float:
    """Lower median of the wall particles' nearest-neighbour distances (host,
    once per case)."""
    if wall.shape[0] < 2:
        return 1.0
    from scipy.spatial import cKDTree
    w = wall.double().numpy()
    d, _ = cKDTree(w).query(w, k=2)
    nn = sorted(d[:, 1].tolist())
    return float(nn[(len(nn) - 1) // 2])


def droplet_impact_case(cfg, *, drop_speed: float = 0.0, label: str = "") -> CaseSpec:
    """The 2-D droplet impact of ``tensorsph.droplet_impact`` (pool plus
    circular drop from ``make_particles``, walls from ``wall_lattice`` up to
    ``domain_top``, droplet_impact.py:666-760) as a ``CaseSpec``; the drop
    starts with the downward speed ``drop_speed`` (the reference drops it from
    rest).  ``surface_tension_coefficient > 0`` turns on the consistent CSF
    force (csf_consistent.py:384-446) with the configuration's curvature
    ("fit_quadratic", "mls" or "fit_circle") and delta_s normalisation
    ("legacy" or "local_range")."""
    from .droplet_impact import domain_top, lattice_mass_unit, make_particles, validate_config, wall_lattice
    validate_config(cfg)
    curvature = {"fit_quadratic": 0, "mls": 1, "fit_circle": 2}
    normalization = {"legacy": 0, "local_range": 1}
    contact = {"rotate": 1, "young": 2, "brackbill": 3}
    if cfg.surface_tension_coefficient > 0.0:
        if cfg.csf_scheme != "consistent":
            raise NotImplementedError("the device engine implements the consistent CSF scheme")
        if cfg.csf_curvature not in curvature or cfg.csf_delta_normalization not in normalization:
            raise ValueError(f"unknown csf_curvature {cfg.csf_curvature!r} or csf_delta_normalization "
                             f"{cfg.csf_delta_normalization!r}")
        if cfg.contact_angle is not None:
            if cfg.contact_angle_model not in contact:
                raise ValueError(f"unknown contact_angle_model {cfg.contact_angle_model!r}")
            if cfg.contact_angle_model == "rotate" and not 0.0 < cfg.contact_angle_reach <= 2.0:
                raise NotImplementedError("the device engine's contact-angle boundary reaches at most 2 h "
                                          "(the wall particles of the list rows)")
    x, mass = make_particles(cfg, "cpu")
    wall = wall_lattice(cfg, "cpu")
    x = x.double().contiguous()
    wall = wall.double().contiguous()
    n_pool = int(((x[:, 1] <= cfg.pool_depth)).sum())
    v = torch.zeros_like(x)
    v[n_pool:, 1] = -float(drop_speed)
    h = cfg.h_factor * cfg.dx
    top = domain_top(cfg)
    allpos = torch.cat((x, wall))
    p = _case_params(dim=2, n_fluid=x.shape[0], n_wall=wall.shape[0], n_obstacle=0, cfg=cfg, h=h,
                     wall_mass=lattice_mass_unit(cfg), box_hi=(cfg.pool_width, top, 0.0),
                     lo=allpos.min(dim=0).values.tolist(), hi=allpos.max(dim=0).values.tolist())
    p.surface_tension = float(cfg.surface_tension_coefficient)
    if p.surface_tension > 0.0:
        p.csf_curvature = curvature[cfg.csf_curvature]
        p.csf_delta_normalization = normalization[cfg.csf_delta_normalization]
        if cfg.contact_angle is not None and wall.shape[0]:
            p.csf_contact_model = contact[cfg.contact_angle_model]
            p.csf_contact_angle = float(cfg.contact_angle)
            p.csf_contact_reach = float(cfg.contact_angle_reach)
            if cfg.contact_angle_model != "rotate":
                # contact_angle_isph.py:75-81 and :104-107: A = (median nearest-
                # neighbour wall spacing)^2, the traction calibration 0.9611
                p.csf_wall_area = _wall_spacing(wall) ** 2
                p.csf_traction_calibration = 0.9611
    return CaseSpec(p, x, v, mass.double().contiguous(), wall, label or "droplet_impact")


def shear_decay_case(n: int, *, box: float = 1.0, amplitude: float = 1.0e-3, nu: float = 1.0e-2,
                     sound_speed: float = 1.0, rho0: float = 1000.0, gamma: float = 7.0,
                     h_factor: float = 1.3, jitter: float = 0.01, seed: int = 0,
                     skin_factor: float = 0.25, courant: float = 0.25, density_diffusion: float = 0.0,
                     density_diffusion_form: str = "antuono", density_diffusion_eigenvalue_floor: float = 0.1,
                     label: str = "") -> CaseSpec:
    """A triply periodic shear decay u_x = A sin(2 pi z / L) on an n^3 lattice
    with a seeded uniform jitter of +-jitter dx, as a ``CaseSpec`` of the batch
    engine (its WCSPH operators: Tait, Morris viscous Laplacian; no gravity, no
    walls).  dt is the smaller of acoustic CFL ``courant`` and 0.9 x the
    viscous limit 0.125 h^2 / nu.  ``density_diffusion`` > 0 adds the density
    diffusion of threed's ``accelerations`` (operators3.py:226-236, scale
    2 delta c0 h), by default its psi form with the renormalised gradient."""
    if density_diffusion_form not in ("antuono", "molteni"):
        raise ValueError(f"unknown density_diffusion_form {density_diffusion_form!r}")
    dx = box / n
    h = h_factor * dx
    dt = min(courant * h / sound_speed, 0.9 * 0.125 * h * h / nu)
    g = torch.Generator().manual_seed(seed)
    ax = torch.arange(n, dtype=torch.float64) * dx
    gx, gy, gz = torch.meshgrid(ax, ax, ax, indexing="ij")
    x = torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), -1)
    x = (x + jitter * dx * (2.0 * torch.rand(x.shape, generator=g, dtype=torch.float64) - 1.0)
         ).remainder(box).contiguous()
    k = 2.0 * math.pi / box
    v = torch.zeros_like(x)
    v[:, 0] = amplitude * torch.sin(k * x[:, 2])
    from .dam_break_3d import mass_3d as _mass3d
    m = torch.full((x.shape[0],), _mass3d(dx, h_factor, rho0, True), dtype=torch.float64)
    p = _lib.CaseParams()
    p.dim, p.n_fluid, p.n_wall, p.n_obstacle = 3, x.shape[0], 0, 0
    p.h, p.rho0, p.sound_speed, p.gamma = h, rho0, sound_speed, gamma
    p.gravity, p.viscosity, p.wall_friction, p.diffusion_scale = 0.0, nu, 0.0, 0.0
    if density_diffusion > 0.0:
        p.diffusion_scale = 2.0 * density_diffusion * sound_speed * h
        p.diffusion_form = 1 if density_diffusion_form == "antuono" else 0
        p.diffusion_eigen_floor = float(density_diffusion_eigenvalue_floor)
    p.dt, p.wall_mass, p.skin = dt, 0.0, skin_factor * h
    for kk in range(3):
        p.box_hi[kk] = box
        p.grid_lo[kk], p.grid_hi[kk] = 0.0, box
    p.tolerance = 0.25 * dx
    p.shift_vref_floor = 0.05 * sound_speed
    p.periodic_box = box
    return CaseSpec(p, x, v, m, torch.zeros((0, 3), dtype=torch.float64), label or "shear_decay_3d")


# ------------------------------------------------------------------ engine --

def _engine_params(max_fluid, max_wall, max_obstacle, max_cells, max_cases, max_neighbors,
                   diag_ring, max_fit_neighbors=0) -> _lib.EngineParams:
    prm = _lib.EngineParams()
    prm.max_fluid, prm.max_wall, prm.max_obstacle = int(max_fluid), int(max_wall), int(max_obstacle)
    prm.max_cells, prm.max_cases = int(max_cells), int(max_cases)
    prm.max_neighbors, prm.diag_ring = int(max_neighbors), int(diag_ring)
    prm.max_fit_neighbors = int(max_fit_neighbors)
    return prm


def engine_bytes(*, max_fluid, max_wall, max_obstacle=0, max_cells, max_cases=1,
                 max_neighbors=160, diag_ring=1024, max_fit_neighbors=0) -> int:
    """Device bytes of an engine with these capacities (its HBM footprint)."""
    prm = _engine_params(max_fluid, max_wall, max_obstacle, max_cells, max_cases, max_neighbors,
                         diag_ring, max_fit_neighbors)
    n = _lib.lib().tsph_engine_bytes(ctypes.byref(prm))
    if n <= 0:
        raise ValueError("invalid engine capacities")
    return int(n)


class BatchEngine:
    """Fixed-capacity device engine holding any number of independent cases."""

    def __init__(self, *, max_fluid: int, max_wall: int, max_obstacle: int = 0, max_cells: int,
                 max_cases: int = 1, max_neighbors: int = 160, diag_ring: int = 1024,
                 max_fit_neighbors: int = 0, device: torch.device | None = None):
        dev = device or _lib.cuda_device()
        self.device = dev
        self.stream = torch.cuda.Stream(device=dev)
        self.capacity = dict(max_fluid=int(max_fluid), max_wall=int(max_wall),
                             max_obstacle=int(max_obstacle), max_cells=int(max_cells),
                             max_cases=int(max_cases), max_neighbors=int(max_neighbors),
                             diag_ring=int(diag_ring), max_fit_neighbors=int(max_fit_neighbors))
        self.params = _engine_params(max_fluid, max_wall, max_obstacle, max_cells, max_cases,
                                     max_neighbors, diag_ring, max_fit_neighbors)
        L = _lib.lib()
        nbytes = L.tsph_engine_bytes(ctypes.byref(self.params))
        if nbytes <= 0:
            raise ValueError("invalid engine capacities")
        self.nbytes = int(nbytes)
        self._handle = ctypes.c_void_p(None)
        self.stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(self.stream):
            self.arena = torch.empty(self.nbytes, dtype=torch.uint8, device=dev)
        _lib.check(L.tsph_engine_create(ctypes.byref(self.params), self.arena.data_ptr(), self.nbytes,
                                        self.stream.cuda_stream, ctypes.byref(self._handle)),
                   "tsph_engine_create")
        self.cases: dict[int, CaseSpec] = {}
        self.steps_of: dict[int, int] = {}

    # ----------------------------------------------------------- admission --
    def usage(self) -> dict:
        u = (ctypes.c_int64 * 5)()
        _lib.check(_lib.lib().tsph_engine_usage(self._handle, u), "tsph_engine_usage")
        return dict(fluid=u[0], wall=u[1], obstacle=u[2], cells=u[3], cases=u[4])

    def graph_stats(self) -> dict:
        """Step graphs instantiated and batch changes absorbed by in-place
        graph updates since the engine was created."""
        out = (ctypes.c_int64 * 2)()
        _lib.check(_lib.lib().tsph_engine_graph_stats(self._handle, out), "tsph_engine_graph_stats")
        return {"instantiations": int(out[0]), "updates": int(out[1])}

    def row_entries(self) -> tuple[int, int]:
        """Entries of the current neighbour rows ``(fluid rows, wall rows)``
        (synchronises the engine stream)."""
        out = (ctypes.c_int64 * 2)()
        _lib.check(_lib.lib().tsph_engine_row_entries(self._handle, out, self.stream.cuda_stream),
                   "tsph_engine_row_entries")
        return int(out[0]), int(out[1])

    def fits(self, spec: CaseSpec) -> bool:
        """Whether ``spec`` fits in the free capacity right now."""
        u = self.usage()
        c = self.capacity
        return (u["cases"] < c["max_cases"] and u["fluid"] + spec.n_fluid <= c["max_fluid"]
                and u["wall"] + spec.n_wall <= c["max_wall"]
                and u["obstacle"] + spec.n_obstacle <= c["max_obstacle"]
                and u["cells"] + spec.cells() <= c["max_cells"])

    def add(self, spec: CaseSpec) -> int:
        """Admit a case; returns its id.  Raises RuntimeError when it does not fit."""
        L = _lib.lib()
        cid = ctypes.c_int64(-1)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):
            X = spec.x.to(self.device, torch.float64).contiguous()
            V = (torch.zeros_like(X) if spec.v is None
                 else spec.v.to(self.device, torch.float64).contiguous())
            M = spec.mass.to(self.device, torch.float64).contiguous()
            W = spec.wall.to(self.device, torch.float64).contiguous() if spec.n_wall else None
        rc = L.tsph_engine_add_case(self._handle, ctypes.byref(spec.params), X.data_ptr(),
                                    V.data_ptr(), M.data_ptr(), W.data_ptr() if W is not None else None,
                                    self.stream.cuda_stream, ctypes.byref(cid))
        if rc == _lib.ERR_CAPACITY:
            raise RuntimeError("the case does not fit in the engine's free capacity")
        _lib.check(rc, "tsph_engine_add_case")
        self.cases[cid.value] = spec
        self.steps_of[cid.value] = 0
        return int(cid.value)

    def remove(self, case_id: int) -> None:
        _lib.check(_lib.lib().tsph_engine_remove_case(self._handle, int(case_id),
                                                      self.stream.cuda_stream),
                   "tsph_engine_remove_case")
        self.cases.pop(case_id, None)
        self.steps_of.pop(case_id, None)

    # ------------------------------------------------------------ stepping --
    def set_block(self, threads: int) -> None:
        """Threads per block of the pair kernels (64, 128 or 256): a tuning knob."""
        _lib.check(_lib.lib().tsph_engine_set_block(self._handle, int(threads)),
                   "tsph_engine_set_block")

    def set_batch(self, depth: int) -> None:
        """Neighbour records in flight per thread (4, 8 or 16): a tuning knob."""
        _lib.check(_lib.lib().tsph_engine_set_batch(self._handle, int(depth)),
                   "tsph_engine_set_batch")

    def step(self, steps: int = 1, graph: bool = True) -> None:
        """Advance every case ``steps`` steps on the engine's stream (no host
        synchronisation)."""
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        L = _lib.lib()
        fn = L.tsph_engine_step if graph else L.tsph_engine_step_eager
        _lib.check(fn(self._handle, int(steps), self.stream.cuda_stream), "tsph_engine_step")
        for k in self.steps_of:
            self.steps_of[k] += int(steps)

    def _hand_over(self, *tensors):
        """Make the caller's current stream wait for the engine stream, so the
        returned tensors are safe to use there."""
        cur = torch.cuda.current_stream(self.device)
        if cur != self.stream:
            cur.wait_stream(self.stream)
            for t in tensors:
                t.record_stream(cur)

    STAGES = ("rebuild", "density", "diffusion_eos", "walls", "force", "reaction",
              "integrate", "shift_rebuild", "concentration", "gradient", "select", "shift_apply")

    def step_timed(self) -> dict:
        """One eager step with CUDA events between stages; ``{stage: ms}``."""
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        ms = (ctypes.c_float * 12)()
        n = ctypes.c_int64(0)
        _lib.check(_lib.lib().tsph_engine_step_timed(self._handle, self.stream.cuda_stream, ms,
                                                     ctypes.byref(n)), "tsph_engine_step_timed")
        for k in self.steps_of:
            self.steps_of[k] += 1
        return {self.STAGES[i]: float(ms[i]) for i in range(n.value)}

    def graph_kernels(self) -> tuple[int, int]:
        """Kernel launches of the captured step graph: ``(every step, per list
        pass that rebuilds)``; the second runs in a conditional node only when
        some case's lists are rebuilt in that pass."""
        k = (ctypes.c_int64 * 2)()
        _lib.check(_lib.lib().tsph_engine_graph_kernels(self._handle, k), "tsph_engine_graph_kernels")
        return int(k[0]), int(k[1])

    # -------------------------------------------------------------- output --
    def diagnostics(self, case_id: int, first: int, count: int) -> torch.Tensor:
        """Per-step meter rows ``(count, len(DIAG_FIELDS))`` of one case."""
        with torch.cuda.stream(self.stream):
            out = torch.empty((count, len(DIAG_FIELDS)), dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib().tsph_engine_diag(self._handle, int(case_id), out.data_ptr(),
                                               int(first), int(count), self.stream.cuda_stream),
                   "tsph_engine_diag")
        self._hand_over(out)
        return out

    def read(self, case_id: int):
        """``(x, v, rho, p)`` of one case's fluid in its original order (device)."""
        spec = self.cases[case_id]
        n, dim = spec.n_fluid, spec.dim
        with torch.cuda.stream(self.stream):
            x = torch.empty((n, dim), dtype=torch.float64, device=self.device)
            v = torch.empty_like(x)
            rho = torch.empty(n, dtype=torch.float64, device=self.device)
            p = torch.empty_like(rho)
        _lib.check(_lib.lib().tsph_engine_read(self._handle, int(case_id), x.data_ptr(),
                                               v.data_ptr(), rho.data_ptr(), p.data_ptr(),
                                               self.stream.cuda_stream), "tsph_engine_read")
        self._hand_over(x, v, rho, p)
        return x, v, rho, p

    def status(self, case_id: int) -> dict:
        buf = (ctypes.c_int64 * 8)()
        rc = _lib.lib().tsph_engine_status(self._handle, int(case_id), buf, self.stream.cuda_stream)
        out = dict(escapes=buf[0], clamps=buf[1], rebuilds=buf[2], steps=buf[3], row_max=buf[4],
                   finished=bool(buf[5]), status=buf[6], final_step=buf[7])
        if rc == _lib.ERR_CAPACITY:
            raise RuntimeError(f"neighbour row capacity exceeded (longest row {buf[4]}); "
                               "raise max_neighbors")
        _lib.check(rc, "tsph_engine_status")
        return out

    def clock(self, case_id: int) -> tuple[float, float]:
        """(elapsed, dt) of an adaptive case after the steps run so far: the
        time at the start of its next step and that step's size before the
        clamp to the target time (synchronises the engine stream)."""
        buf = (ctypes.c_double * 2)()
        _lib.check(_lib.lib().tsph_engine_clock(self._handle, int(case_id), buf, self.stream.cuda_stream),
                   "tsph_engine_clock")
        return float(buf[0]), float(buf[1])

    def close(self) -> None:
        if self._handle is not None and self._handle.value:
            torch.cuda.synchronize(self.device)
            _lib.lib().tsph_engine_destroy(self._handle)
            self._handle = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def capacity_for(specs, *, max_neighbors: int = 160, diag_ring: int = 1024, cases: int | None = None):
    """Capacities that hold every case of ``specs`` at once."""
    specs = list(specs)
    csf = any(s.dim == 2 and s.params.surface_tension > 0.0 for s in specs)
    return dict(max_fluid=sum(s.n_fluid for s in specs), max_wall=max(1, sum(s.n_wall for s in specs)),
                max_obstacle=sum(s.n_obstacle for s in specs),
                max_cells=sum(s.cells() for s in specs),
                max_cases=cases if cases is not None else len(specs),
                max_neighbors=max_neighbors, diag_ring=diag_ring,
                max_fit_neighbors=FIT_NEIGHBORS if csf else 0)


# ------------------------------------------------------- single-case engine --

@dataclass
class DamBreak3DRun:
    """Run record with the fields of the reference ``DamBreak3DRun`` that the
    engine measures (dam_break_3d.py:488-549) plus the obstacle force series."""

    times: list
    front: list
    kinetic_energy: list
    potential_energy: list
    mass: float
    escaped: int
    rebuilds: int
    max_speed: float
    max_density_compression: float
    initial_mass: float
    final_mass: float
    final_positions: torch.Tensor
    initial_energy: float = 0.0
    final_energy: float = 0.0
    steps_taken: int = 0
    simulated_time: float = 0.0
    obstacle_force: list = field(default_factory=list)
    obstacle_impulse: list = field(default_factory=list)   # SPH force impulse [x, y, z], N s
    clamp_impulse: list = field(default_factory=list)      # obstacle clamp impulse [x, y, z], N s
    obstacle_clamps: int = 0
    snapshots: list = field(default_factory=list)
    tvc_log: list = field(default_factory=list)
    resumed: bool = False
    dt_min: float = 0.0              # smallest and largest step of the run
    dt_max: float = 0.0
    max_acoustic_courant: float = 0.0

    @property
    def mass_drift(self) -> float:
        return self.final_mass - self.initial_mass


class DamBreak3DEngine(BatchEngine):
    """One device-resident 3-D dam-break case (a batch of one, sized to it)."""

    def __init__(self, cfg: DamBreak3DConfig, *, obstacle=None, shift_every: int = 0,
                 seed: int | None = None, max_neighbors: int = 160, diag_ring: int = 8192,
                 device: torch.device | None = None, host_state=None, velocity=None,
                 first_step: int = 0, start_clock=None):
        spec = dam_break_3d_case(cfg, obstacle=obstacle, shift_every=shift_every, seed=seed,
                                 host_state=host_state, velocity=velocity, first_step=first_step,
                                 start_clock=start_clock)
        super().__init__(**capacity_for([spec], max_neighbors=max_neighbors, diag_ring=diag_ring),
                         device=device)
        self.cfg = cfg
        self.spec = spec
        self.n_fluid, self.n_wall, self.n_obstacle = spec.n_fluid, spec.n_wall, spec.n_obstacle
        self.case_id = self.add(spec)
        self.state_bytes = (spec.x.numel() + spec.mass.numel() + spec.wall.numel()) * 8

    @functools.cached_property
    def initial_mass(self) -> float:
        return float(self.spec.mass.sum())

    @functools.cached_property
    def initial_pe(self) -> float:
        return float((self.spec.mass * self.cfg.gravity * self.spec.x[:, 1]).sum())

    @property
    def steps_done(self) -> int:
        return self.steps_of.get(self.case_id, 0)

    build_host_state = staticmethod(dam_break_3d_host_state)

    def diagnostics(self, first: int, count: int) -> torch.Tensor:  # type: ignore[override]
        return super().diagnostics(self.case_id, first, count)

    def state(self):
        """``(x, v, rho, p)`` of the fluid in the original particle order (device)."""
        return self.read(self.case_id)

    def status(self) -> dict:  # type: ignore[override]
        return super().status(self.case_id)


def pick_trial(trials: list[dict], tolerance: float = 0.01) -> dict:
    """The tuner's choice among timed trials (``skin_factor``, ``ms_per_step``,
    ...).  The trials start from rest, where no list is rebuilt yet: a larger
    skin costs longer rows, which they time, and saves rebuilds once the flow
    moves, which they cannot; so among the trials within ``tolerance`` of the
    fastest the largest skin wins, then the fastest at it."""
    fastest = min(t["ms_per_step"] for t in trials)
    close = [t for t in trials if t["ms_per_step"] <= (1.0 + tolerance) * fastest]
    widest = max(t["skin_factor"] for t in close)
    return min((t for t in close if t["skin_factor"] == widest), key=lambda t: t["ms_per_step"])


def tune_single_case(cfg: DamBreak3DConfig, *, obstacle=None, shift_every: int = 0, host_state=None,
                     skins=(0.1, 0.15, 0.25), blocks=(128, 256), batches=(4, 8, 16), steps: int = 60,
                     device=None, cache: bool = True) -> dict:
    """Autotune one 3-D case by timing: the Verlet skin (which sets the cell edge
    2h + skin and how often lists are rebuilt), the pair kernels' block size and
    their batch depth.  Each trial runs ``steps`` graph steps on the device
    (rebuilds included); the results do not depend on the choice beyond the
    summation order of the skin pairs.  Returns the fastest and every trial;
    with ``cache`` a previous result for the same workload and GPU
    (``tensorsph_b200.tuning``) is returned without timing, and a new one kept."""
    from dataclasses import replace
    from . import tuning
    key = None
    if cache:
        n = host_state[0].shape[0] if host_state is not None else dam_break_3d_host_state(cfg, obstacle)[0].shape[0]
        dev = device or torch.device("cuda", torch.cuda.current_device())
        key = tuning.tuning_key("dam_break_3d" + ("+obstacle" if obstacle is not None else "")
                                + f"+shift{shift_every}", dim=3, particles=n, h_over_dx=cfg.h_factor,
                                candidates={"skins": skins, "blocks": blocks, "batches": batches},
                                gpu=torch.cuda.get_device_name(dev))
        hit = tuning.lookup(key)
        if hit is not None:
            return {"best": hit, "trials": [], "cached": True}
    trials = []
    for skin in skins:
        c = replace(cfg, pair_skin_factor=float(skin))
        eng = DamBreak3DEngine(c, obstacle=obstacle, shift_every=shift_every, host_state=host_state,
                               diag_ring=8, device=device)
        eng.step(3)
        for block in blocks:
            for batch in batches:
                eng.set_block(block)
                eng.set_batch(batch)
                eng.step(2)
                start = torch.cuda.Event(enable_timing=True)
                stop = torch.cuda.Event(enable_timing=True)
                start.record(eng.stream)
                eng.step(steps)
                stop.record(eng.stream)
                stop.synchronize()
                trials.append({"skin_factor": float(skin), "block": block, "batch": batch,
                               "ms_per_step": start.elapsed_time(stop) / steps})
        eng.close()
    best = pick_trial(trials)
    if key is not None:
        tuning.store(key, best)
    return {"best": best, "trials": trials, "cached": False}


def _sample_steps(steps: int, output_every: int, dt: float):
    """``(step, elapsed)`` of the reference loops' sample points: every
    ``output_every`` steps and the last, with ``elapsed`` accumulated step by
    step as the loops do (dam_break_3d.py:617-705, dam_break.py:365-461)."""
    out, elapsed = [], 0.0
    for k in range(steps + 1):
        if k % output_every == 0 or k == steps:
            out.append((k, elapsed))
        elapsed += dt
    return out


def _snapshot_plan(snapshot_times, samples):
    """``(step, elapsed)`` of each requested snapshot: a target time is taken at
    the first sample point whose time reaches it (several targets may share
    one), as dam_break_3d.py:658-664 does."""
    targets = sorted(float(t) for t in (snapshot_times or []))
    plan, nxt = [], 0
    for k, t in samples:
        while nxt < len(targets) and t >= targets[nxt] - 1.0e-12:
            plan.append((k, t))
            nxt += 1
    return plan


class _Snapshots:
    """Positions and velocities of one case copied to pinned host memory on a
    side stream: the engine's stream only runs the read kernel, and the copies
    overlap the steps that follow."""

    def __init__(self, eng, case_id):
        self.eng, self.case_id = eng, case_id
        self.side = torch.cuda.Stream(device=eng.device)
        self.taken = []

    def take(self, elapsed: float):
        with torch.cuda.stream(self.side):
            x, v, _, _ = self.eng.read(self.case_id)
            hx = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
            hv = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
            hx.copy_(x, non_blocking=True)
            hv.copy_(v, non_blocking=True)
        self.taken.append((elapsed, hx, hv))

    def result(self) -> list:
        self.side.synchronize()
        return list(self.taken)


def _run_with_snapshots(eng, case_id, steps: int, plan) -> list:
    """Advance ``steps`` steps, taking the planned snapshots on the way."""
    snaps = _Snapshots(eng, case_id)
    done = 0
    for k, t in plan:
        if k > done:
            eng.step(k - done)
            done = k
        snaps.take(t)
    if steps > done:
        eng.step(steps - done)
    return snaps.result()


def _tvc_log(cfg, diag, n_fluid: int, first: int = 0, upto: int | None = None) -> list:
    """The reference's per-application log of the transport-velocity
    correction (dam_break_3d.py:697-704) from the meter rows ``diag`` of
    steps ``first, first + 1, ...``: steps k = tvc_every, 2 tvc_every, ...
    below ``upto`` (default ``cfg.steps``) and from ``first`` on."""
    every = int(getattr(cfg, "tvc_every", 0) or 0)
    if not every:
        return []
    upto = cfg.steps if upto is None else upto
    adaptive = bool(getattr(cfg, "adaptive_dt", False))   # times from the rows
    h = cfg.h_factor * cfg.dx
    out, elapsed = [], 0.0
    for k in range(upto):
        if k >= first and k > 0 and k % every == 0:
            row = diag[k - first]
            out.append({"step": k, "time": float(row[25]) if adaptive else elapsed,
                        "max_shift_over_h": float(row[16]) / h,
                        "mean_shift_over_h": float(row[17]) / n_fluid / h,
                        "kept_fraction": (None if cfg.tvc_scope_tol is None
                                          else float(row[18]) / n_fluid),
                        "clipped_fraction": float(row[19]) / n_fluid})
        elapsed += cfg.dt
    return out


def _elapsed_after(steps: int, dt: float) -> list:
    """``out[k]``: simulated time at the start of step k, accumulated step by
    step as the reference loops do."""
    out, elapsed = [0.0], 0.0
    for _ in range(steps + 1):
        elapsed += dt
        out.append(elapsed)
    return out


class _DeviceRecord:
    """Series, maxima, counters and impulses of a 3-D device run through a
    global step, from the meter rows of steps ``first, first + 1, ...`` and,
    for a resumed run, the checkpoint it resumed from (whose series cover the
    steps before ``first``)."""

    def __init__(self, cfg, samples, first: int, prev: dict | None, n_fluid: int, initial_energy: float):
        self.cfg, self.samples, self.first, self.n_fluid = cfg, samples, first, n_fluid
        self.prev = prev or {}
        self.dev = self.prev.get("device_run", {})
        self.initial_energy = float(self.dev.get("initial_energy", initial_energy))

    def collect(self, rows, upto: int) -> dict:
        """Everything through global step ``upto``: samples and maxima over
        rows ``first..upto``, forces, counters and impulses through the last
        integrated step ``min(upto, steps - 1)``."""
        cfg, first, prev, dev = self.cfg, self.first, self.prev, self.dev
        rows = torch.as_tensor(rows)
        new = [(k, t) for k, t in self.samples if first <= k <= upto]
        last = min(upto, cfg.steps - 1) - first  # row of the last integrated step (< 0: none)

        def series(key, col):
            return list(prev.get(key, dev.get(key, []))) + [float(rows[k - first, col]) for k, _ in new]

        out = {
            "times": list(prev.get("times", [])) + [t for _, t in new],
            "front": series("front", 2),
            "kinetic_energy": list(dev.get("kinetic_energy", [])) + [float(rows[k - first, 6]) for k, _ in new],
            "potential_energy": list(dev.get("potential_energy", [])) + [float(rows[k - first, 7]) for k, _ in new],
            "speed_samples": list(dev.get("speed_samples", [])) + [float(rows[k - first, 1]) for k, _ in new],
            "obstacle_force": list(dev.get("obstacle_force", [])) + (rows[:last + 1, 3:6].tolist() if last >= 0 else []),
            "tvc_log": list(dev.get("tvc_log", [])) + _tvc_log(cfg, rows, self.n_fluid, first, min(upto + 1, cfg.steps)),
        }
        imp = [float(v) for v in prev.get("sph_impulse", [0.0, 0.0, 0.0])]
        cimp = [float(v) for v in prev.get("clamp_impulse", [0.0, 0.0, 0.0])]
        escapes, clamps, rebuilds = int(prev.get("escapes", 0)), int(prev.get("clamps", 0)), int(dev.get("rebuilds", 0))
        if last >= 0:
            r = rows[last]
            imp = [imp[0] + float(r[14]), imp[1] + float(r[20]), imp[2] + float(r[21])]
            cimp = [cimp[i] + float(r[22 + i]) for i in range(3)]
            escapes, clamps, rebuilds = escapes + int(r[8]), clamps + int(r[9]), rebuilds + int(r[10])
        seen = rows[:upto - first + 1]
        speeds = float(prev.get("speeds", 0.0))
        compression = float(prev.get("compression", -1.0))
        if seen.shape[0]:
            speeds = max(speeds, float(seen[:, 1].max()))
            compression = max(compression, float(seen[:, 0].max()) / cfg.rho0 - 1.0)
        out.update(sph_impulse=imp, clamp_impulse=cimp, escapes=escapes, clamps=clamps, rebuilds=rebuilds,
                   speeds=speeds, compression=compression)
        return out

    def payload(self, rows, step: int) -> dict:
        """What the checkpoint after the update of ``step`` stores."""
        r = self.collect(rows, step)
        keep = ("kinetic_energy", "potential_energy", "speed_samples", "obstacle_force", "tvc_log", "rebuilds")
        extra = {"device_run": {**{k: r[k] for k in keep}, "initial_energy": self.initial_energy}}
        return {**r, "dt": self.cfg.dt, "extra": extra}


def run_case(cfg: DamBreak3DConfig, pair_skin_factor: float | None = None, snapshot_times=None,
             seed: int | None = None, *, obstacle=None, shift_every: int = 0,
             max_neighbors: int = 160, checkpoint_path=None, checkpoint_every: int = 0,
             resume: bool = True) -> DamBreak3DRun:
    """Integrate the 3-D dam break on the GPU and return the run record.

    Same loop as dam_break_3d.py:569-734: ``cfg.steps`` steps of ``cfg.dt``,
    meters sampled every ``cfg.output_every`` steps and at the end.  The whole
    loop stays on the device; meters come back once at the end.
    ``snapshot_times`` fills ``run.snapshots`` with ``(time, positions,
    velocities)`` at the first sample point reaching each time, copied to the
    host while the loop goes on.

    Checkpoints follow kleefsman_obstacle_3d.py:553-706: with
    ``checkpoint_path`` naming an existing file and ``resume`` the run
    continues from it (a file of another configuration or particle count is
    refused); with ``checkpoint_every > 0`` the state after the update of
    every step k with ``k % checkpoint_every == 0`` is written there in that
    case's format (by ``CheckpointWriter``, off the step loop); a completed
    run removes the file.  A resumed run rebuilds its neighbour lists at the
    resume step, so it agrees with an uninterrupted one to round-off.
    """
    from pathlib import Path
    from .checkpoint import CheckpointWriter, load_checkpoint
    if pair_skin_factor is not None:
        from dataclasses import replace
        cfg = replace(cfg, pair_skin_factor=pair_skin_factor)
    host = dam_break_3d_host_state(cfg, obstacle, seed)
    prev = None
    if checkpoint_path is not None and resume and Path(checkpoint_path).exists():
        prev = load_checkpoint(checkpoint_path, cfg, obstacle)
        if tuple(prev["positions"].shape) != tuple(host[0].shape):
            raise ValueError(f"checkpoint holds {tuple(prev['positions'].shape)} particles, "
                             f"this configuration builds {tuple(host[0].shape)}")
        if "device_run" not in prev:
            raise ValueError("checkpoint carries no device run record; it was written by another driver")
        if not cfg.adaptive_dt and prev["step"] + 1 > cfg.steps:
            raise ValueError(f"checkpoint step {prev['step']} is not below the run's {cfg.steps} steps")
        if cfg.adaptive_dt and prev["elapsed"] >= cfg.steps * cfg.dt - 1.0e-12 * max(1.0, cfg.steps * cfg.dt):
            raise ValueError(f"checkpoint time {prev['elapsed']} is not below the run's {cfg.steps * cfg.dt}")
    if cfg.adaptive_dt:
        return _run_3d_adaptive(cfg, obstacle, shift_every, seed, max_neighbors, snapshot_times, host=host,
                                prev=prev, checkpoint_path=checkpoint_path, checkpoint_every=checkpoint_every)
    first = prev["step"] + 1 if prev else 0
    if prev:
        host = (prev["positions"].double(), host[1], host[2], host[3])
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=shift_every, seed=seed,
                           max_neighbors=max_neighbors, diag_ring=max(cfg.steps + 2, 2), host_state=host,
                           velocity=prev["velocity"] if prev else None, first_step=first)
    samples = _sample_steps(cfg.steps, cfg.output_every, cfg.dt)
    record = _DeviceRecord(cfg, samples, first, prev, eng.n_fluid, eng.initial_pe)
    writer = None
    if checkpoint_path is not None and checkpoint_every > 0:
        writer = CheckpointWriter(eng, eng.case_id, checkpoint_path, cfg, obstacle=obstacle)
    # (steps done, kind, arg): a snapshot before the update of its sample
    # step, a checkpoint after the update of its step
    events = [(k, 0, t) for k, t in _snapshot_plan(snapshot_times, samples) if k >= first]
    if writer is not None:
        events += [(k + 1, 1, k) for k in range(first, cfg.steps) if k % checkpoint_every == 0]
    events.sort(key=lambda e: (e[0], e[1]))
    after = _elapsed_after(cfg.steps, cfg.dt)
    snaps = _Snapshots(eng, eng.case_id)
    done = first
    try:
        for at, kind, arg in events:
            if at > done:
                eng.step(at - done)
                done = at
            if kind == 0:
                snaps.take(arg)
            else:
                writer.take(arg, after[arg + 1], first, arg - first + 1,
                            lambda rows, k=arg: record.payload(rows, k))
        if cfg.steps > done:
            eng.step(cfg.steps - done)
        snapshots = snaps.result()
        with torch.cuda.stream(eng.stream):
            x, v, rho, p = eng.state()
            xs, vs = x.cpu(), v.cpu()
        eng.status()
        # the reference evaluates the right-hand side once more at step == steps
        # to record the final meters, without integrating it
        eng.step(1)
        with torch.cuda.stream(eng.stream):
            diag = eng.diagnostics(first, cfg.steps + 1 - first).cpu()
        if writer is not None:
            writer.close()
    finally:
        if writer is not None and writer.thread is not None:
            writer.thread.join()
    rec = record.collect(diag, cfg.steps)
    run = DamBreak3DRun(
        times=rec["times"], front=rec["front"], kinetic_energy=rec["kinetic_energy"],
        potential_energy=rec["potential_energy"], mass=eng.initial_mass, escaped=rec["escapes"],
        rebuilds=rec["rebuilds"], max_speed=rec["speeds"],
        max_density_compression=rec["compression"], initial_mass=eng.initial_mass,
        final_mass=eng.initial_mass, final_positions=xs, initial_energy=record.initial_energy,
        steps_taken=cfg.steps, simulated_time=cfg.steps * cfg.dt, obstacle_force=rec["obstacle_force"],
        obstacle_impulse=rec["sph_impulse"], clamp_impulse=rec["clamp_impulse"],
        obstacle_clamps=rec["clamps"], snapshots=snapshots, tvc_log=rec["tvc_log"], resumed=prev is not None,
        dt_min=cfg.dt, dt_max=cfg.dt,
        max_acoustic_courant=cfg.dt * (cfg.sound_speed + rec["speeds"]) / (cfg.h_factor * cfg.dx))
    masses = eng.spec.mass
    run.final_energy = float(0.5 * (masses[:, None] * vs.square()).sum()
                             + (masses * cfg.gravity * xs[:, 1]).sum())
    eng.close()
    if checkpoint_path is not None:
        # a completed run must not be resumed by the next attempt
        try:
            Path(checkpoint_path).unlink()
        except FileNotFoundError:
            pass
    return run


class _AdaptiveRecord(_DeviceRecord):
    """``_DeviceRecord`` of an adaptive run: its samples are the
    output_every-th steps and the final one, their times read from the meter
    rows (column 25, the time at the step's start), and its last integrated
    step is the one before the final step (or ``upto`` while the run goes on)."""

    def __init__(self, cfg, first: int, prev: dict | None, n_fluid: int, initial_energy: float):
        super().__init__(cfg, [], first, prev, n_fluid, initial_energy)
        self.base_cfg = cfg

    def collect(self, rows, upto: int, final: int | None = None) -> dict:  # type: ignore[override]
        from dataclasses import replace
        rows_t = torch.as_tensor(rows)
        every = max(1, int(self.base_cfg.output_every))
        self.samples = [(k, float(rows_t[k - self.first, 25])) for k in range(self.first, upto + 1)
                        if k % every == 0 or k == final]
        self.cfg = replace(self.base_cfg, steps=final if final is not None else upto + 1)
        out = super().collect(rows, upto)
        seen = rows_t[:upto - self.first + 1]
        dev = self.dev
        # smallest and largest step before its clamp to the target time, and the
        # acoustic Courant peak of the steps taken (dam_break.py:394-397)
        h = self.base_cfg.h_factor * self.base_cfg.dx
        lo = [float(seen[:, 27].min())] if seen.shape[0] else []
        hi = [float(seen[:, 27].max())] if seen.shape[0] else []
        cour = [float((seen[:, 26] * (self.base_cfg.sound_speed + seen[:, 1])).max()) / h] if seen.shape[0] else []
        out["dt_min"] = min([float(dev["dt_min"])] + lo) if "dt_min" in dev else (lo[0] if lo else self.base_cfg.dt)
        out["dt_max"] = max([float(dev["dt_max"])] + hi) if "dt_max" in dev else (hi[0] if hi else self.base_cfg.dt)
        out["courant"] = max([float(dev.get("courant", 0.0))] + cour)
        out["rebuilds"] = int(dev.get("rebuilds", 0)) + (int(seen[-1, 10]) if seen.shape[0] else 0)
        return out

    def payload(self, rows, step: int, dt: float) -> dict:  # type: ignore[override]
        """What the checkpoint after the update of ``step`` stores; ``dt`` is
        the size next_dt gave the step after it."""
        r = self.collect(rows, step)
        keep = ("kinetic_energy", "potential_energy", "speed_samples", "obstacle_force", "tvc_log", "rebuilds",
                "dt_min", "dt_max", "courant")
        extra = {"device_run": {**{k: r[k] for k in keep}, "initial_energy": self.initial_energy}}
        return {**r, "dt": float(dt), "extra": extra}


def _run_3d_adaptive(cfg, obstacle, shift_every: int, seed, max_neighbors: int, snapshot_times=None, *,
                     host=None, prev=None, checkpoint_path=None, checkpoint_every: int = 0) -> DamBreak3DRun:
    """The 3-D loop with adaptive_dt (dam_break_3d.py:617-711): meters at
    every output_every-th step and at the final one, times from the device.

    With checkpoints (kleefsman_obstacle_3d.py:598-640) the state after the
    update of every step k with ``k % checkpoint_every == 0`` is written with
    the loop's clock (the time at the start of step k + 1 and next_dt's step
    for it); a run resumed from ``prev`` starts its engine at step
    ``prev["step"] + 1`` with that clock and continues the series."""
    from pathlib import Path
    from .checkpoint import CheckpointWriter
    host = host if host is not None else dam_break_3d_host_state(cfg, obstacle, seed)
    first = prev["step"] + 1 if prev else 0
    if prev:
        host = (prev["positions"].double(), host[1], host[2], host[3])
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=shift_every, seed=seed,
                           max_neighbors=max_neighbors, diag_ring=4 * cfg.steps + 1100, host_state=host,
                           velocity=prev["velocity"] if prev else None, first_step=first,
                           start_clock=(prev["elapsed"], prev["dt"]) if prev else None)
    record = _AdaptiveRecord(cfg, first, prev, eng.n_fluid, eng.initial_pe)
    writer = None
    if checkpoint_path is not None and checkpoint_every > 0:
        writer = CheckpointWriter(eng, eng.case_id, checkpoint_path, cfg, obstacle=obstacle)

    def checkpoint(k):
        elapsed, dt = eng.clock(eng.case_id)
        writer.take(k, elapsed, first, k - first + 1, lambda rows: record.payload(rows, k, dt))

    try:
        final, snapshots = _advance_adaptive(eng, eng.case_id, cfg, snapshot_times=snapshot_times or [],
                                             first=first, start_time=prev["elapsed"] if prev else 0.0,
                                             checkpoint_every=checkpoint_every if writer else 0,
                                             on_checkpoint=checkpoint if writer else None)
        with torch.cuda.stream(eng.stream):
            x, v, _, _ = eng.state()
            xs, vs = x.cpu(), v.cpu()
            diag = eng.diagnostics(first, final + 1 - first).cpu()
        if writer is not None:
            writer.close()
    finally:
        if writer is not None and writer.thread is not None:
            writer.thread.join()
    rec = record.collect(diag, final, final=final)
    run = DamBreak3DRun(
        times=rec["times"], front=rec["front"], kinetic_energy=rec["kinetic_energy"],
        potential_energy=rec["potential_energy"], mass=eng.initial_mass, escaped=rec["escapes"],
        rebuilds=rec["rebuilds"], max_speed=rec["speeds"], max_density_compression=rec["compression"],
        initial_mass=eng.initial_mass, final_mass=eng.initial_mass, final_positions=xs,
        initial_energy=record.initial_energy, steps_taken=final, simulated_time=float(diag[final - first, 25]),
        obstacle_force=rec["obstacle_force"], obstacle_impulse=rec["sph_impulse"],
        clamp_impulse=rec["clamp_impulse"], obstacle_clamps=rec["clamps"], tvc_log=rec["tvc_log"],
        snapshots=snapshots, dt_min=rec["dt_min"], dt_max=rec["dt_max"],
        max_acoustic_courant=rec["courant"], resumed=prev is not None)
    masses = eng.spec.mass
    run.final_energy = float(0.5 * (masses[:, None] * vs.square()).sum()
                             + (masses * cfg.gravity * xs[:, 1]).sum())
    eng.close()
    if checkpoint_path is not None:
        # a completed run must not be resumed by the next attempt
        try:
            Path(checkpoint_path).unlink()
        except FileNotFoundError:
            pass
    return run


@dataclass
class DamBreakRun:
    """The fields of the reference 2-D ``DamBreakRun`` (dam_break.py:250-280)
    that the device loop measures."""

    times: list
    front: list
    kinetic_energy: list
    potential_energy: list
    mass: float
    escaped: int
    rebuilds: int
    max_speed: float
    max_density_compression: float
    final_positions: torch.Tensor
    steps_taken: int = 0
    simulated_time: float = 0.0
    snapshots: list = field(default_factory=list)
    max_tvc_shift: float = 0.0       # largest |shift| of one correction, m
    max_tvc_clipped: float = 0.0     # largest fraction of fluid one correction clipped
    dt_min: float = 0.0              # smallest and largest step of the run
    dt_max: float = 0.0
    max_acoustic_courant: float = 0.0


def _max_courant(cfg, diag) -> float:
    """max over the steps of dt (c0 + |v|max) / h (dam_break.py:394-397)."""
    h = cfg.h_factor * cfg.dx
    return max(float(diag[k, 26]) * (cfg.sound_speed + float(diag[k, 1])) / h for k in range(diag.shape[0]))


def _advance_adaptive(eng, cid, cfg, chunk: int = 64, snapshot_times=None, *, first: int = 0,
                      start_time: float = 0.0, checkpoint_every: int = 0, on_checkpoint=None):
    """Step an adaptive case until it records its final meters (the step at
    which the simulated time reaches steps * dt); returns that step, and with
    ``snapshot_times`` also the snapshots.  Steps after the final one leave
    the case as it is.

    A snapshot target is taken at the first sample step (every
    ``output_every``-th and the final one) whose starting time reaches it, as
    dam_break.py:409-414 does: the chunks then end on the sample steps, and
    the time at the start of step k is read from the meter row of step k-1.
    A run resumed at step ``first`` (its clock at ``start_time``) skips the
    targets before that time.  With ``checkpoint_every`` the chunks also end
    after each integrated step k with ``k % checkpoint_every == 0``, where
    ``on_checkpoint(k)`` is called."""
    max_steps = 4 * cfg.steps + 1000
    targets = sorted(float(t) for t in (snapshot_times or []) if first == 0 or float(t) >= start_time - 1.0e-12)
    snaps, nxt = [], 0

    def take(t):
        nonlocal nxt
        while nxt < len(targets) and t >= targets[nxt] - 1.0e-12:
            with torch.cuda.stream(eng.stream):
                x, v = eng.read(cid)[:2]
                snaps.append((t, x.cpu(), v.cpu()))
            nxt += 1

    every = max(1, int(cfg.output_every)) if targets else chunk
    if first % every == 0:
        take(start_time)
    done = first
    while done <= max_steps:
        n = min(every - done % every, max_steps + 1 - done)
        if checkpoint_every:
            # end the chunk after the next checkpoint step k >= done
            k = done + (-done) % checkpoint_every
            n = min(n, k + 1 - done)
        eng.step(n)
        done += n
        st = BatchEngine.status(eng, cid)
        if st["finished"]:
            final = int(st["final_step"])
            if targets:
                with torch.cuda.stream(eng.stream):
                    take(float(BatchEngine.diagnostics(eng, cid, final, 1).cpu()[0, 25]))
            return (final, snaps) if snapshot_times is not None else final
        if checkpoint_every and (done - 1) % checkpoint_every == 0:
            on_checkpoint(done - 1)
        if nxt < len(targets) and done % every == 0:
            with torch.cuda.stream(eng.stream):
                row = BatchEngine.diagnostics(eng, cid, done - 1, 1).cpu()[0]
            take(float(row[25]) + float(row[26]))
    raise RuntimeError(f"the adaptive run did not reach {cfg.steps * cfg.dt} s in {max_steps} steps")


def _run_2d_adaptive(cfg, max_neighbors: int, snapshot_times=None) -> "DamBreakRun":
    """The 2-D loop with adaptive_dt (dam_break.py:367-465): meters at every
    output_every-th step and at the final one, times from the device."""
    spec = dam_break_2d_case(cfg, shift_every=cfg.shift_every)
    eng = BatchEngine(**capacity_for([spec], max_neighbors=max_neighbors, diag_ring=4 * cfg.steps + 1100))
    cid = eng.add(spec)
    final, snapshots = _advance_adaptive(eng, cid, cfg, snapshot_times=snapshot_times or [])
    with torch.cuda.stream(eng.stream):
        x = eng.read(cid)[0].cpu()
        diag = eng.diagnostics(cid, 0, final + 1).cpu()
    sample = [k for k in range(final + 1) if k % cfg.output_every == 0 or k == final]
    dts = diag[:, 27]
    run = DamBreakRun(times=[float(diag[k, 25]) for k in sample], front=[float(diag[k, 2]) for k in sample],
                      kinetic_energy=[float(diag[k, 6]) for k in sample],
                      potential_energy=[float(diag[k, 7]) for k in sample],
                      mass=float(spec.mass.sum()), escaped=int(diag[final - 1, 8]) if final else 0,
                      rebuilds=int(diag[final, 10]), max_speed=float(diag[:, 1].max()),
                      max_density_compression=float(diag[:, 0].max()) / cfg.rho0 - 1.0,
                      final_positions=x, steps_taken=final, simulated_time=float(diag[final, 25]),
                      snapshots=snapshots, dt_min=float(dts.min()), dt_max=float(dts.max()),
                      max_acoustic_courant=_max_courant(cfg, diag))
    every = int(cfg.tvc_every or 0)
    applied = [k for k in range(1, final) if every and k % every == 0]
    if applied:
        run.max_tvc_shift = max(float(diag[k, 16]) for k in applied)
        run.max_tvc_clipped = max(float(diag[k, 19]) for k in applied) / spec.n_fluid
    eng.close()
    return run


def run_dam_break_2d(cfg, *, snapshot_times=None, max_neighbors: int = 64) -> DamBreakRun:
    """Integrate the 2-D dam break (dam_break.py:319-460 with the pair cache,
    fixed dt) on the GPU and return the measured trajectory;
    ``snapshot_times`` as in ``run_case``.  Shifting and the transport-velocity
    correction (``tvc_every``, scopes "all", "bulk_g" and "bulk", the
    ``truncated_linear`` limiter, the clip) each run, not both together."""
    if cfg.adaptive_dt:
        return _run_2d_adaptive(cfg, max_neighbors, snapshot_times)
    spec = dam_break_2d_case(cfg, shift_every=cfg.shift_every)
    eng = BatchEngine(**capacity_for([spec], max_neighbors=max_neighbors,
                                     diag_ring=max(cfg.steps + 1, 1)))
    cid = eng.add(spec)
    samples = _sample_steps(cfg.steps, cfg.output_every, cfg.dt)
    snapshots = _run_with_snapshots(eng, cid, cfg.steps, _snapshot_plan(snapshot_times, samples))
    with torch.cuda.stream(eng.stream):
        x = eng.read(cid)[0].cpu()
    # the reference evaluates the right-hand side once more at step == steps
    # to record the final meters, without integrating it
    eng.step(1)
    with torch.cuda.stream(eng.stream):
        diag = eng.diagnostics(cid, 0, cfg.steps + 1).cpu()
    st = eng.status(cid)
    sample = [k for k, _ in samples]
    run = DamBreakRun(times=[t for _, t in samples], front=[float(diag[k, 2]) for k in sample],
                      kinetic_energy=[float(diag[k, 6]) for k in sample],
                      potential_energy=[float(diag[k, 7]) for k in sample],
                      mass=float(spec.mass.sum()), escaped=int(st["escapes"]),
                      rebuilds=int(st["rebuilds"]),
                      max_speed=float(diag[:, 1].max()),
                      max_density_compression=float(diag[:, 0].max()) / cfg.rho0 - 1.0,
                      final_positions=x, steps_taken=cfg.steps,
                      simulated_time=cfg.steps * cfg.dt, snapshots=snapshots,
                      dt_min=cfg.dt, dt_max=cfg.dt,
                      max_acoustic_courant=_max_courant(cfg, diag))
    every = int(cfg.tvc_every or 0)
    applied = [k for k in range(1, cfg.steps) if every and k % every == 0]
    if applied:
        run.max_tvc_shift = max(float(diag[k, 16]) for k in applied)
        run.max_tvc_clipped = max(float(diag[k, 19]) for k in applied) / spec.n_fluid
    eng.close()
    return run
