"""2-D delta-plus SPH step on the GPU (``tensorsph.delta_plus``).

``delta_plus_step`` keeps the reference signature, checks, exceptions and
``DeltaPlusStep`` result (delta_plus.py:19-229): Wendland C2 at h = 2 dx,
linear EOS, fixed-ghost wall pressure with gravity, pressure + Monaghan radial
viscosity + slip-wall forces, continuity with the wall flux, psi-form density
diffusion through the eigen-floored first-moment inverse, the Marrone
empty-cap interface band and the regularised, wall-tangent positional shift
-- all in ``csrc/delta_plus.cu`` over one symmetric gather list.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
import math
import weakref

import torch

from . import _lib
from .droplet_impact import symmetric_rows
from .neighbor_search import grid_pairs

__all__ = ["DeltaPlusStep", "delta_plus_step", "delta_plus_step3"]


# The gather rows of the last pair list a step was given: a Verlet cache
# (PairListCache) hands back the same tensor between rebuilds, so a caller
# that steps with it pays for the check and the row build once per rebuild.
# The rows are dropped with the pair list they were built from.
_ROWS: dict = {"pairs": None, "version": None, "nrows": None, "rows": None}


def _forget_rows(_ref=None) -> None:
    _ROWS.update(pairs=None, version=None, nrows=None, rows=None)


def _rows_of(pairs: torch.Tensor, dev, nrows: int):
    ref = _ROWS["pairs"]
    if (ref is not None and ref() is pairs and _ROWS["version"] == pairs._version
            and _ROWS["nrows"] == nrows):
        return _ROWS["rows"]
    i, j = pairs.unbind(1)
    if bool(((i < 0) | (i >= j) | (j >= nrows)).any()):
        raise ValueError("each pair must have 0 <= i < j < number of particles")
    _forget_rows()
    rows = symmetric_rows(_lib.to_dev(pairs, dev), nrows)
    _ROWS.update(pairs=weakref.ref(pairs, _forget_rows), version=pairs._version, nrows=nrows, rows=rows)
    return rows


@dataclass
class DeltaPlusStep:
    position: torch.Tensor
    velocity: torch.Tensor
    density: torch.Tensor
    acceleration: torch.Tensor
    wall_reaction: torch.Tensor
    shift: torch.Tensor


def delta_plus_step(pos, velocity, density, mass, *, dx, sound_speed, reference_speed,
                    dt, rho0=1000., gravity=9.81, viscosity=1.e-6, diffusion=.1, alpha=.02,
                    wall=None, wall_velocity=None, wall_normal=None, pairs=None):
    """Advance an equal-spacing 2-D liquid by one delta-plus step (h = 2 dx)."""
    return _delta_plus(2, pos, velocity, density, mass, dx=dx, sound_speed=sound_speed,
                       reference_speed=reference_speed, dt=dt, rho0=rho0, gravity=gravity,
                       viscosity=viscosity, diffusion=diffusion, alpha=alpha, wall=wall,
                       wall_velocity=wall_velocity, wall_normal=wall_normal, pairs=pairs)


def delta_plus_step3(pos, velocity, density, mass, *, dx, sound_speed, reference_speed,
                     dt, rho0=1000., gravity=9.81, viscosity=1.e-6, diffusion=.1, alpha=.02,
                     wall=None, wall_velocity=None, wall_normal=None, pairs=None):
    """The delta-plus step of ``delta_plus_step`` for a 3-D liquid (y up).

    The reference's step is 2-D only (delta_plus.py:119); this is the same
    sequence of statements in 3-D: the 3-D Wendland C2 constant
    21 / (16 pi h^3) (threed/kernel3.py:139-164), the radial viscous stress
    coefficient 2 (D + 2) nu = 10 nu (and its time-step limit dt nu_r / 10 <=
    h^2 / 8), wall stations of volume dx^3, the 3 x 3 first moment, the
    empty-cap test's tangential distance |ray x n|, and a wall-tangent shift
    that conflicts with the interface normal reduced to its part along
    n_wall x n_surface instead of to zero.  Arguments, checks, exceptions and
    the ``DeltaPlusStep`` result are the 2-D step's with (N, 3) arrays."""
    return _delta_plus(3, pos, velocity, density, mass, dx=dx, sound_speed=sound_speed,
                       reference_speed=reference_speed, dt=dt, rho0=rho0, gravity=gravity,
                       viscosity=viscosity, diffusion=diffusion, alpha=alpha, wall=wall,
                       wall_velocity=wall_velocity, wall_normal=wall_normal, pairs=pairs)


def _delta_plus(dim, pos, velocity, density, mass, *, dx, sound_speed, reference_speed,
                dt, rho0, gravity, viscosity, diffusion, alpha, wall, wall_velocity, wall_normal,
                pairs):
    if (pos.ndim != 2 or pos.shape[1] != dim or velocity.shape != pos.shape
            or density.shape != pos.shape[:1] or mass.shape != density.shape
            or not len(pos) or pos.dtype not in (torch.float32, torch.float64)):
        raise ValueError(f"expected a nonempty {dim}-D fluid and one density and mass per particle")
    if not all(math.isfinite(x) for x in (dx, sound_speed, reference_speed, dt,
                                          rho0, gravity, viscosity, diffusion, alpha)):
        raise ValueError("solver parameters must be finite")
    if min(dx, sound_speed, dt, rho0) <= 0 or min(reference_speed, viscosity, diffusion, alpha) < 0:
        raise ValueError("invalid length, speed, density, step or transport coefficient")
    h = 2 * dx
    coef = 2 * (dim + 2)   # Monaghan's radial viscous stress, 8 in 2-D
    radial_viscosity = coef * viscosity + alpha * h * sound_speed
    if (dt * sound_speed > .3 * h or dt * radial_viscosity / coef > .125 * h * h
            or dt * diffusion * sound_speed > .125 * h):
        raise ValueError("time step exceeds an acoustic, viscous or diffusive limit")
    if wall is None:
        wall = pos.new_empty((0, dim))
    if wall_velocity is None:
        wall_velocity = torch.zeros_like(wall)
    if wall.ndim != 2 or wall.shape[1] != dim or wall_velocity.shape != wall.shape:
        raise ValueError(f"expected matching (W, {dim}) wall positions and velocities")
    if wall_normal is None and len(wall) == 0:
        wall_normal = wall
    if wall_normal is None or wall_normal.shape != wall.shape:
        raise ValueError("provide a wall_normal per ghost station for free slip")
    if any(x.dtype != pos.dtype or x.device != pos.device
           for x in (velocity, density, mass, wall, wall_velocity, wall_normal)):
        raise ValueError("states must share a floating dtype and device")
    if not bool(((density > 0) & (mass > 0) & density.isfinite() & mass.isfinite()).all()):
        raise ValueError("density and mass must be positive and finite")
    norms = wall_normal.norm(dim=1)
    if not bool((norms.isfinite() & (norms > 0)).all()):
        raise ValueError("wall normals must be finite and nonzero")
    if not all(bool(x.isfinite().all()) for x in (pos, velocity, wall, wall_velocity)):
        raise ValueError("particle positions and velocities must be finite")
    n, nw = pos.shape[0], wall.shape[0]
    out_device = pos.device
    dev = _lib.cuda_device(pos)
    dtype = pos.dtype
    P, V, R, M = (_lib.to_dev(t.detach(), dev, dtype).contiguous() for t in (pos, velocity, density, mass))
    W, WV, WN = (_lib.to_dev(t.detach(), dev, dtype).contiguous() for t in (wall, wall_velocity, wall_normal))
    if pairs is None:
        cloud = torch.cat((P, W)) if nw else P
        pairs_dev, _, _ = grid_pairs(cloud, 2 * h) if n + nw >= 2 else (
            torch.zeros((0, 2), dtype=torch.long, device=dev), 0, None)
        rowptr, entries = symmetric_rows(pairs_dev, n + nw)
    else:
        if pairs.ndim != 2 or pairs.shape[1] != 2 or pairs.dtype != torch.long:
            raise ValueError("expected a (P, 2) long pair list")
        if pairs.device != pos.device:
            raise ValueError("pair list must share the device of the state")
        rowptr, entries = _rows_of(pairs, dev, n + nw)
    prm = _lib.DeltaPlusParams()
    prm.dtype, prm.n_fluid, prm.n_wall = _lib.dtype_code(dtype), n, nw
    prm.dx, prm.sound_speed, prm.reference_speed, prm.dt = float(dx), float(sound_speed), \
        float(reference_speed), float(dt)
    prm.rho0, prm.gravity, prm.viscosity = float(rho0), float(gravity), float(viscosity)
    prm.diffusion, prm.alpha = float(diffusion), float(alpha)
    prm.dim = dim
    out_pos = torch.empty_like(P)
    out_vel = torch.empty_like(P)
    out_rho = torch.empty_like(R)
    acc = torch.empty_like(P)
    reaction = torch.zeros_like(W)
    shift = torch.empty_like(P)
    status = ctypes.c_int(0)
    ptr = lambda t: t.data_ptr() if t.numel() else None  # noqa: E731
    io = _lib.DeltaPlusIO(P.data_ptr(), V.data_ptr(), R.data_ptr(), M.data_ptr(), ptr(W), ptr(WV),
                          ptr(WN), rowptr.data_ptr(), entries.data_ptr(), out_pos.data_ptr(),
                          out_vel.data_ptr(), out_rho.data_ptr(), acc.data_ptr(), ptr(reaction),
                          shift.data_ptr(), ctypes.cast(ctypes.pointer(status), ctypes.c_void_p))
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_delta_plus_workspace_bytes(ctypes.byref(prm)), dev)
    rc = L.tsph_delta_plus_step(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                                _lib.stream(dev))
    if rc == _lib.ERR_STATE:
        if status.value & 1:
            raise FloatingPointError("nonpositive extrapolated wall density")
        raise FloatingPointError("δ⁺-SPH density became nonpositive or nonfinite")
    _lib.check(rc, "tsph_delta_plus_step")
    to = lambda t: t.to(out_device)  # noqa: E731
    return DeltaPlusStep(to(out_pos), to(out_vel), to(out_rho), to(acc), to(reaction), to(shift))
