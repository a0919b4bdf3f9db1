"""3-D WCSPH operators on the GPU (``tensorsph.threed.operators3``).

``accelerations`` keeps the reference signature and its ``(acc, rho,
pressure)`` return order (operators3.py:212-256): summation density,
optional diffusive term (Antuono psi form by default, Molteni on request),
Tait EOS without the ratio floor, Adami wall pressure, the symmetric pressure
force and the second-moment renormalised Brookshaw viscosity (order 2 or 4),
all in the fused kernels of ``csrc/threed.cu``.
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib
from ..droplet_impact import symmetric_rows
from .neighbors3 import _box_list

__all__ = ["accelerations", "tait_pressure", "tait_density"]


def tait_pressure(rho, rho0, sound_speed, gamma):
    stiffness = rho0 * sound_speed ** 2 / gamma
    return (stiffness * ((rho / rho0).pow(gamma) - 1.0)).clamp_min(0.0)


def tait_density(pressure, rho0, sound_speed, gamma):
    stiffness = rho0 * sound_speed ** 2 / gamma
    return rho0 * (1.0 + pressure.clamp_min(0.0) / stiffness).pow(1.0 / gamma)


def _params(n, nf, dtype, h, *, rho0, sound_speed, gamma, viscosity, gravity, box, renormalise,
            wall_model, viscous_order, density_diffusion, dt, density_diffusion_form,
            density_diffusion_eigenvalue_floor):
    prm = _lib.ThreedParams()
    prm.dtype, prm.n, prm.n_fluid = _lib.dtype_code(dtype), n, nf
    if gravity is not None:
        g = torch.as_tensor(gravity, dtype=torch.float64).reshape(-1).tolist()
        prm.has_gravity = 1
        for k in range(3):
            prm.gravity[k] = g[k]
    if box is not None:
        prm.periodic = 1
        for k, b in enumerate(_box_list(box, 3)):
            prm.box[k] = b
    prm.renormalise = int(bool(renormalise))
    prm.wall_model = 0 if wall_model == "adami" else 1
    prm.viscous_order = int(viscous_order)
    prm.diffusion_form = 1 if density_diffusion_form == "antuono" else 0
    prm.h, prm.rho0, prm.sound_speed, prm.gamma = float(h), rho0, sound_speed, gamma
    prm.viscosity = float(viscosity)
    prm.diffusion = float(density_diffusion)
    prm.dt = float(dt) if dt is not None else 0.0
    prm.eigen_floor = float(density_diffusion_eigenvalue_floor)
    return prm


def _run_rows(prm, P, V, M, rowptr, entries, acc=None, rho=None, pressure=None):
    """One pass of ``tsph_threed_accelerations`` over prepared gather rows
    (device tensors); outputs may be passed in to be overwritten."""
    n, dev, dtype = int(prm.n), P.device, P.dtype
    acc = torch.empty((n, 3), dtype=dtype, device=dev) if acc is None else acc
    rho = torch.empty(n, dtype=dtype, device=dev) if rho is None else rho
    pressure = torch.empty(n, dtype=dtype, device=dev) if pressure is None else pressure
    io = _lib.ThreedIO(P.data_ptr(), V.data_ptr(), M.data_ptr(), rowptr.data_ptr(),
                       entries.data_ptr(), acc.data_ptr(), rho.data_ptr(), pressure.data_ptr())
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_threed_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_threed_accelerations(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(),
                                           ws.numel(), _lib.stream(dev)),
               "tsph_threed_accelerations")
    return acc, rho, pressure


def accelerations(pos, vel, mass, h, pairs, *, rho0, sound_speed, gamma=7.0, viscosity=0.0,
                  gravity=None, box=None, n_fluid=None, renormalise=True, wall_model="adami",
                  viscous_order=2, density_diffusion=0.0, dt=None,
                  density_diffusion_form="antuono", density_diffusion_eigenvalue_floor=0.1):
    """Right-hand side of a 3-D fluid (+ static wall) set; ``(acc, rho, pressure)``."""
    n = pos.shape[0]
    nf = n if n_fluid is None else int(n_fluid)
    if density_diffusion > 0.0 and (dt is None or dt <= 0.0):
        raise ValueError("density_diffusion > 0 requires a positive dt")
    if nf < n and wall_model not in ("adami", "tait"):
        raise ValueError(f"unknown wall_model {wall_model!r}")
    if density_diffusion > 0.0 and density_diffusion_form not in ("molteni", "antuono"):
        raise ValueError(f"unknown density_diffusion_form {density_diffusion_form!r}")
    if viscous_order not in (2, 4):
        raise ValueError("viscous_order must be 2 or 4")
    if pos.shape[1] != 3:
        raise ValueError("accelerations implements 3-D clouds")
    out_device = pos.device
    dev = _lib.cuda_device(pos)
    dtype = pos.dtype
    P = _lib.to_dev(pos.detach(), dev)
    V = _lib.to_dev(vel.detach(), dev, dtype)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    rowptr, entries = symmetric_rows(_lib.to_dev(pairs, dev), n)
    prm = _params(n, nf, dtype, h, rho0=rho0, sound_speed=sound_speed, gamma=gamma,
                  viscosity=viscosity, gravity=gravity, box=box, renormalise=renormalise,
                  wall_model=wall_model, viscous_order=viscous_order,
                  density_diffusion=density_diffusion, dt=dt,
                  density_diffusion_form=density_diffusion_form,
                  density_diffusion_eigenvalue_floor=density_diffusion_eigenvalue_floor)
    acc, rho, pressure = _run_rows(prm, P, V, M, rowptr, entries)
    return acc.to(out_device), rho.to(out_device), pressure.to(out_device)
