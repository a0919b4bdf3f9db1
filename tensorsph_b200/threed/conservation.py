"""Conservation meters (``tensorsph.threed.conservation``) on the GPU.

``diagnostics`` keeps the reference signature and row
(threed/conservation.py:104-121) and computes every sum in one FP64 device
reduction (``tsph_meters``): mass, linear and angular momentum, kinetic
energy, Tait internal energy and the centre of mass, with the circular mean in
a periodic box.  The single-quantity helpers read the same reduction;
``internal_energy`` is the per-particle field (``tsph_internal_energy``).
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib

__all__ = ["mass_total", "momentum", "angular_momentum", "kinetic_energy", "internal_energy",
           "total_energy", "centre_of_mass", "diagnostics", "relative_drift"]


def _meters(pos, vel, mass, rho=None, *, rho0=1.0, sound_speed=1.0, gamma=7.0,
            periodic_box=None, origin=None) -> torch.Tensor:
    if pos.ndim != 2 or pos.shape[1] not in (2, 3):
        raise ValueError("pos must be (N, 2) or (N, 3)")
    if vel.shape != pos.shape or mass.shape != pos.shape[:1]:
        raise ValueError("vel must match pos and mass must be (N,)")
    if rho is not None and rho.shape != mass.shape:
        raise ValueError("rho must be (N,)")
    n, dim = pos.shape
    dev = _lib.cuda_device(pos)
    dtype = pos.dtype
    P = _lib.to_dev(pos.detach(), dev)
    V = _lib.to_dev(vel.detach(), dev, dtype)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    R = _lib.to_dev(rho.detach(), dev, dtype) if rho is not None else None
    prm = _lib.MeterParams()
    prm.dim, prm.dtype, prm.n = dim, _lib.dtype_code(dtype), n
    prm.rho0, prm.sound_speed, prm.gamma = float(rho0), float(sound_speed), float(gamma)
    if origin is not None:
        o = torch.as_tensor(origin, dtype=torch.float64).reshape(-1).tolist()
        for k in range(dim):
            prm.origin[k] = o[k]
    if periodic_box is not None:
        b = torch.as_tensor(periodic_box, dtype=torch.float64).reshape(-1)
        b = b.expand(dim) if b.numel() == 1 else b
        prm.periodic = 1
        for k in range(dim):
            prm.box[k] = float(b[k])
    out = torch.empty(13, dtype=torch.float64, device=dev)
    io = _lib.MeterIO(P.data_ptr(), V.data_ptr(), M.data_ptr(), R.data_ptr() if R is not None else None,
                      out.data_ptr())
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_meters_workspace_bytes(), dev)
    _lib.check(L.tsph_meters(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                             _lib.stream(dev)), "tsph_meters")
    return out.cpu()


def mass_total(mass: torch.Tensor) -> float:
    z = torch.zeros((mass.shape[0], 3), dtype=mass.dtype, device=mass.device)
    return float(_meters(z, z, mass)[0])


def momentum(mass: torch.Tensor, vel: torch.Tensor) -> torch.Tensor:
    m = _meters(torch.zeros_like(vel), vel, mass)
    return m[1:1 + vel.shape[1]].to(vel.dtype)


def angular_momentum(mass: torch.Tensor, pos: torch.Tensor, vel: torch.Tensor,
                     origin=None) -> torch.Tensor:
    if pos.shape[1] != 3:
        raise ValueError("angular momentum needs 3-D vectors")
    return _meters(pos, vel, mass, origin=origin)[4:7].to(pos.dtype)


def kinetic_energy(mass: torch.Tensor, vel: torch.Tensor) -> float:
    return float(_meters(torch.zeros_like(vel), vel, mass)[7])


def internal_energy(rho: torch.Tensor, rho0: float, sound_speed: float,
                    gamma: float) -> torch.Tensor:
    dev = _lib.cuda_device(rho)
    R = _lib.to_dev(rho.detach(), dev)
    out = torch.empty_like(R)
    _lib.check(_lib.lib().tsph_internal_energy(R.data_ptr(), R.numel(), _lib.dtype_code(R.dtype),
                                               float(rho0), float(sound_speed), float(gamma),
                                               out.data_ptr(), _lib.stream(dev)),
               "tsph_internal_energy")
    return out.to(rho.device)


def total_energy(mass: torch.Tensor, vel: torch.Tensor, rho: torch.Tensor,
                 rho0: float, sound_speed: float, gamma: float) -> float:
    return float(_meters(torch.zeros_like(vel), vel, mass, rho, rho0=rho0,
                         sound_speed=sound_speed, gamma=gamma)[9])


def centre_of_mass(mass: torch.Tensor, pos: torch.Tensor, periodic_box=None) -> torch.Tensor:
    m = _meters(pos, torch.zeros_like(pos), mass, periodic_box=periodic_box)
    return m[10:10 + pos.shape[1]].to(pos.dtype)


def diagnostics(pos: torch.Tensor, vel: torch.Tensor, mass: torch.Tensor,
                rho: torch.Tensor, *, rho0: float, sound_speed: float,
                gamma: float = 7.0, periodic_box=None, origin=None) -> dict:
    """One row of the conservation ledger (one device reduction)."""
    m = _meters(pos, vel, mass, rho, rho0=rho0, sound_speed=sound_speed, gamma=gamma,
                periodic_box=periodic_box, origin=origin)
    d = pos.shape[1]
    p = m[1:1 + d]
    return {
        "mass": float(m[0]),
        "momentum": p.tolist(),
        "momentum_magnitude": float(torch.linalg.vector_norm(p)),
        "angular_momentum": m[4:7].tolist(),
        "kinetic_energy": float(m[7]),
        "internal_energy": float(m[8]),
        "total_energy": float(m[9]),
        "centre_of_mass": m[10:10 + d].tolist(),
    }


def relative_drift(values, *, scale: float | None = None) -> dict:
    """Drift of a scalar series (threed/conservation.py:124-146): first and last
    value, their difference, the largest magnitude, and the difference relative
    to ``scale`` (default |first|) and to that largest magnitude -- host
    arithmetic on the ledger's floats."""
    series = [float(v) for v in values]
    start, end = series[0], series[-1]
    largest = max(abs(v) for v in series)
    denom = abs(float(scale)) if scale is not None else abs(start)
    change = end - start
    return {"initial": start, "final": end, "delta": change, "peak_abs": largest, "scale": denom,
            "relative_drift": change / denom if denom > 0.0 else None,
            "relative_to_peak": change / largest if largest > 0.0 else None}
