"""Triply periodic shear-wave decay on the GPU (``tensorsph.threed.solver``).

``run_shear_wave`` keeps the reference signature and result
(threed/solver.py:211-308): the double-shear field u_x = A sin(k y) sin(k z)
on a cubic lattice, kick-drift-kick with the periodic wrap, a Verlet-skin
periodic pair list rebuilt when 2 max|x - x_ref| (minimum image) exceeds the
skin, the ``accelerations`` right-hand side, and every ``sample_every`` steps
the mode amplitude and a conservation row.  Everything per step runs on the
device: the pair search (``grid_pairs``), the gather rows (built once per
rebuild), the operator pass, the KDK halves (``tsph_kick_drift``), the
displacement test and the meters.  The only host read per step is the
displacement scalar that decides a rebuild, as in the reference.

``run_shear_decay`` is the single-mode variant u_x = A sin(k z) with a seeded
uniform jitter of the lattice, the projection 2 <u_x sin(k z)> and the
analytic decay rate nu k^2 of that mode.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
import math

import torch

from .. import _lib
from ..droplet_impact import symmetric_rows
from ..neighbor_search import grid_pairs, max_displacement
from . import conservation
from .kernel3 import calibrated_particle_mass
from .operators3 import _params, _run_rows
from .solver import acoustic_dt, cubic_lattice

__all__ = ["ShearWaveResult", "run_shear_wave", "run_shear_decay", "fit_decay_rate",
           "mode_amplitude", "analytic_mode_decay", "shear_wave_field", "cell_dx",
           "wavenumber_for"]


def mode_amplitude(pos: torch.Tensor, vel: torch.Tensor, wavenumber: float, mode: int = 0) -> float:
    """Projection of v_x on sin(k y) sin(k z) (mode 0, operators3.py:401-408) or
    on sin(k z) (mode 1); one FP64 device reduction."""
    dev = _lib.cuda_device(pos)
    P = _lib.to_dev(pos.detach(), dev)
    V = _lib.to_dev(vel.detach(), dev, P.dtype)
    out = torch.empty((), dtype=torch.float64, device=dev)
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_meters_workspace_bytes(), dev)
    _lib.check(L.tsph_mode_amplitude(P.data_ptr(), V.data_ptr(), P.shape[0], _lib.dtype_code(P.dtype),
                                     float(wavenumber), int(mode), ws.data_ptr(), ws.numel(),
                                     out.data_ptr(), _lib.stream(dev)), "tsph_mode_amplitude")
    return float(out)


def analytic_mode_decay(nu: float, wavenumber: float) -> float:
    """Decay exponent of u = A sin(ky) sin(kz): 2 nu k^2 (operators3.py:411-413)."""
    return 2.0 * nu * wavenumber ** 2


def shear_wave_field(pos: torch.Tensor, amplitude: float, wavenumber: float) -> torch.Tensor:
    """u_x = A sin(k y) sin(k z) (operators3.py:416-421), set up on the host."""
    vel = torch.zeros_like(pos)
    vel[:, 0] = amplitude * torch.sin(wavenumber * pos[:, 1]) * torch.sin(wavenumber * pos[:, 2])
    return vel


def cell_dx(box: float, n: int) -> float:
    return float(box) / float(n)


def wavenumber_for(box: float, periods: int = 1) -> float:
    return 2.0 * math.pi * periods / float(box)


def fit_decay_rate(times, amplitudes) -> float:
    """Least-squares slope of -ln|a| against t without the first sample
    (threed/solver.py:311-327); host arithmetic on the sampled series."""
    t = [float(x) for x in times[1:]]
    a = [abs(float(x)) for x in amplitudes[1:]]
    keep = [(ti, math.log(ai)) for ti, ai in zip(t, a) if ai > 0.0]
    if len(keep) < 2:
        return float("nan")
    tm = sum(k[0] for k in keep) / len(keep)
    lm = sum(k[1] for k in keep) / len(keep)
    num = sum((ti - tm) * (li - lm) for ti, li in keep)
    den = sum((ti - tm) ** 2 for ti, _ in keep)
    return -num / den


@dataclass
class ShearWaveResult:
    """Outcome of one shear-wave run (fields of threed/solver.py:129-208)."""

    n: int
    dx: float
    h: float
    nu: float
    wavenumber: float
    sound_speed: float
    amplitude0: float
    dt: float
    steps: int
    renormalise: bool
    viscous_order: int = 2
    times: list = field(default_factory=list)
    amplitudes: list = field(default_factory=list)
    fit_rate: float = float("nan")
    analytic_rate: float = float("nan")
    diagnostics: list = field(default_factory=list)
    pairs_last: int = 0
    pair_rebuilds: int = 0
    momentum_scale: float = 0.0
    final_positions: torch.Tensor | None = None
    final_velocity: torch.Tensor | None = None
    final_density: torch.Tensor | None = None

    @property
    def rate_error(self) -> float:
        return (self.fit_rate - self.analytic_rate) / self.analytic_rate


def _integrate(pos, vel, mass, *, box, h, nu, rho0, sound_speed, gamma, dt, steps, sample_every,
               skin_factor, renormalise, viscous_order, wavenumber, mode, result, pair_dtype=None):
    """KDK loop.  The state (pos, vel) stays in its own dtype; with
    ``pair_dtype`` set (FP32 on an FP64 state) the operator pass runs on a
    rounded copy of the state each step and its accelerations are applied in
    the state's precision."""
    dev = pos.device
    n = pos.shape[0]
    dtype = pos.dtype if pair_dtype is None else pair_dtype
    mixed = dtype != pos.dtype
    mass_p = mass.to(dtype)
    cutoff = 2.0 * h * (1.0 + skin_factor)
    skin = cutoff - 2.0 * h
    boxes = [float(box)] * 3
    box_arr = (ctypes.c_double * 3)(*boxes)
    prm = _params(n, n, dtype, h, rho0=rho0, sound_speed=sound_speed, gamma=gamma, viscosity=nu,
                  gravity=None, box=box, renormalise=renormalise, wall_model="adami",
                  viscous_order=viscous_order, density_diffusion=0.0, dt=None,
                  density_diffusion_form="antuono", density_diffusion_eigenvalue_floor=0.1)
    L = _lib.lib()
    s = _lib.stream(dev)

    def build(p):
        pairs, _, _ = grid_pairs(p, cutoff, box=boxes)
        rowptr, entries = symmetric_rows(pairs, n)
        return pairs.shape[0], rowptr, entries

    npairs, rowptr, entries = build(pos)
    reference = pos.clone()
    rebuilds = 1
    acc = torch.empty((n, 3), dtype=dtype, device=dev)
    rho = torch.empty(n, dtype=dtype, device=dev)
    prs = torch.empty(n, dtype=dtype, device=dev)
    acc_state = torch.empty((n, 3), dtype=pos.dtype, device=dev) if mixed else acc

    def operator_pass():
        if mixed:
            _run_rows(prm, pos.to(dtype), vel.to(dtype), mass_p, rowptr, entries, acc, rho, prs)
            acc_state.copy_(acc)
        else:
            _run_rows(prm, pos, vel, mass_p, rowptr, entries, acc, rho, prs)

    operator_pass()
    for k in range(steps + 1):
        if k % sample_every == 0:
            result.times.append(k * dt)
            result.amplitudes.append(mode_amplitude(pos, vel, wavenumber, mode))
            result.diagnostics.append(conservation.diagnostics(
                pos, vel, mass, rho.to(pos.dtype), rho0=rho0, sound_speed=sound_speed,
                gamma=gamma, periodic_box=box))
        if k == steps:
            break
        _lib.check(L.tsph_kick_drift(pos.data_ptr(), vel.data_ptr(), acc_state.data_ptr(), n, 3,
                                     _lib.dtype_code(pos.dtype), float(dt), 1, box_arr, s),
                   "tsph_kick_drift")
        moved = float(max_displacement(pos, reference, box=boxes))
        if 2.0 * moved > skin:
            npairs, rowptr, entries = build(pos)
            reference.copy_(pos)
            rebuilds += 1
        operator_pass()
        _lib.check(L.tsph_kick_drift(None, vel.data_ptr(), acc_state.data_ptr(), n, 3,
                                     _lib.dtype_code(pos.dtype), float(dt), 0, None, s),
                   "tsph_kick_drift")
    result.pairs_last = int(npairs)
    result.pair_rebuilds = rebuilds
    result.fit_rate = fit_decay_rate(result.times, result.amplitudes)
    result.final_positions, result.final_velocity, result.final_density = pos, vel, rho
    return result


def run_shear_wave(*, n: int = 16, box: float = 1.0, h_factor: float = 1.3,
                   periods: int = 1, nu: float = 0.02, amplitude: float = 0.1,
                   sound_speed: float = 10.0, rho0: float = 1000.0,
                   gamma: float = 7.0, t_end: float | None = None,
                   dt: float | None = None, steps: int | None = None,
                   sample_every: int = 10, skin_factor: float = 0.25,
                   renormalise: bool = True, viscous_order: int = 2,
                   dtype=torch.float64, device=None) -> ShearWaveResult:
    """The double-shear decay of threed/solver.py:211-308 on the GPU."""
    dx = box / n
    h = h_factor * dx
    wavenumber = 2.0 * math.pi * periods / box
    rate = analytic_mode_decay(nu, wavenumber)
    if t_end is None:
        t_end = 2.0 / rate
    if dt is None:
        dt = acoustic_dt(dx, h, sound_speed)
    if steps is None:
        steps = int(math.ceil(t_end / dt))
    viscous_limit = 0.125 * h * h / max(nu, 1.0e-30)
    if dt > viscous_limit:
        raise ValueError(f"dt = {dt:.3e} s exceeds the viscous limit 0.125 h^2/nu = "
                         f"{viscous_limit:.3e} s")
    if wavenumber * h > 0.9:
        raise ValueError(f"k h = {wavenumber * h:.2f}: the kernel cannot represent this mode")
    dev = device or _lib.cuda_device()
    pos = cubic_lattice((n, n, n), dx, dtype=dtype)
    mass = torch.full((pos.shape[0],), calibrated_particle_mass(dx, h, rho0), dtype=dtype)
    vel = shear_wave_field(pos, amplitude, wavenumber)
    result = ShearWaveResult(n=n, dx=dx, h=h, nu=nu, wavenumber=wavenumber,
                             sound_speed=sound_speed, amplitude0=amplitude, dt=dt, steps=steps,
                             renormalise=renormalise, viscous_order=viscous_order)
    result.momentum_scale = float((mass.unsqueeze(-1) * vel.abs()).sum())
    result.analytic_rate = rate
    return _integrate(pos.to(dev), vel.to(dev), mass.to(dev), box=box, h=h, nu=nu, rho0=rho0,
                      sound_speed=sound_speed, gamma=gamma, dt=dt, steps=steps,
                      sample_every=sample_every, skin_factor=skin_factor,
                      renormalise=renormalise, viscous_order=viscous_order,
                      wavenumber=wavenumber, mode=0, result=result)


def run_shear_decay(*, n: int = 64, box: float = 1.0, h_factor: float = 1.3, amplitude: float = 1e-3,
                    nu: float = 1e-2, sound_speed: float = 1.0, rho0: float = 1000.0,
                    gamma: float = 7.0, steps: int = 2000, dt: float | None = None,
                    jitter: float = 0.01, seed: int = 0, sample_every: int = 20,
                    skin_factor: float = 0.25, renormalise: bool = True, viscous_order: int = 2,
                    dtype=torch.float32, state_dtype=torch.float64,
                    device=None) -> ShearWaveResult:
    """u_x = A sin(2 pi z / L) on an n^3 lattice with a seeded uniform jitter of
    +-jitter dx, minimum-image pairs, KDK at acoustic CFL 0.25; the mode decays
    as exp(-nu k^2 t).  ``dtype`` is the pair arithmetic, ``state_dtype`` the
    positions, velocities and integration (FP64 by default: FP32 pairs on an
    FP64 state)."""
    dx = box / n
    h = h_factor * dx
    k = 2.0 * math.pi / box
    if dt is None:
        dt = acoustic_dt(dx, h, sound_speed)
    if dt > 0.125 * h * h / nu:
        raise ValueError("dt exceeds the viscous limit 0.125 h^2/nu")
    g = torch.Generator().manual_seed(seed)
    pos = cubic_lattice((n, n, n), dx, dtype=torch.float64)
    pos = (pos + jitter * dx * (2.0 * torch.rand(pos.shape, generator=g, dtype=torch.float64) - 1.0)
           ).remainder(box)
    mass = torch.full((pos.shape[0],), calibrated_particle_mass(dx, h, rho0), dtype=torch.float64)
    vel = torch.zeros_like(pos)
    vel[:, 0] = amplitude * torch.sin(k * pos[:, 2])
    result = ShearWaveResult(n=n, dx=dx, h=h, nu=nu, wavenumber=k, sound_speed=sound_speed,
                             amplitude0=amplitude, dt=dt, steps=steps, renormalise=renormalise,
                             viscous_order=viscous_order)
    result.momentum_scale = float((mass.unsqueeze(-1) * vel.abs()).sum())
    result.analytic_rate = nu * k * k
    dev = device or _lib.cuda_device()
    sd = state_dtype if state_dtype is not None else dtype
    return _integrate(pos.to(dev, sd), vel.to(dev, sd), mass.to(dev, sd), box=box, h=h,
                      nu=nu, rho0=rho0, sound_speed=sound_speed, gamma=gamma, dt=dt, steps=steps,
                      sample_every=sample_every, skin_factor=skin_factor, renormalise=renormalise,
                      viscous_order=viscous_order, wavenumber=k, mode=1, result=result,
                      pair_dtype=dtype)
