"""Oracle (test infrastructure only): conservation meters and pair-list density.

numpy restatement of
* threed/conservation.py:41-121 -- mass, momentum, angular momentum, kinetic
  energy, Tait internal energy (:71-85), total energy, centre of mass with the
  circular mean in a periodic box (:88-109);
* droplet_impact.py:761-788 -- ``density_from_neighbor_pairs``: m_i W(0) plus
  the pair sums with the 2-D cubic normalisation.
Sums are taken in FP64 (the device meters' precision).
"""
from __future__ import annotations

import math

import numpy as np

from .pairpass import cubic_kernel


def internal_energy(rho, rho0, sound_speed, gamma):
    ratio = np.asarray(rho, dtype=np.float64) / rho0
    return (sound_speed ** 2 / gamma) * ((ratio ** (gamma - 1.0) - 1.0) / (gamma - 1.0)
                                         + 1.0 / ratio - 1.0)


def centre_of_mass(mass, pos, periodic_box=None):
    m = np.asarray(mass, dtype=np.float64)
    x = np.asarray(pos, dtype=np.float64)
    if periodic_box is None:
        return (m[:, None] * x).sum(0) / m.sum()
    box = np.broadcast_to(np.asarray(periodic_box, dtype=np.float64).reshape(-1), (x.shape[1],))
    ang = 2.0 * math.pi * x / box
    w = m / m.sum()
    mean = np.arctan2((w[:, None] * np.sin(ang)).sum(0), (w[:, None] * np.cos(ang)).sum(0))
    return np.mod(mean / (2.0 * math.pi), 1.0) * box


def diagnostics(pos, vel, mass, rho, *, rho0, sound_speed, gamma=7.0, periodic_box=None,
                origin=None):
    m = np.asarray(mass, dtype=np.float64)
    x = np.asarray(pos, dtype=np.float64)
    v = np.asarray(vel, dtype=np.float64)
    o = np.zeros(x.shape[1]) if origin is None else np.asarray(origin, dtype=np.float64)
    p = (m[:, None] * v).sum(0)
    r = x - o
    if x.shape[1] == 3:
        ang = (m[:, None] * np.cross(r, v)).sum(0)
    else:
        ang = np.array([0.0, 0.0, (m * (r[:, 0] * v[:, 1] - r[:, 1] * v[:, 0])).sum()])
    ke = 0.5 * (m[:, None] * v * v).sum()
    ie = (m * internal_energy(rho, rho0, sound_speed, gamma)).sum()
    return {"mass": m.sum(), "momentum": p, "angular_momentum": ang, "kinetic_energy": ke,
            "internal_energy": ie, "total_energy": ke + ie,
            "centre_of_mass": centre_of_mass(m, x, periodic_box)}


def density_from_neighbor_pairs(pos, mass, h, pairs):
    T = pos.dtype.type
    n = pos.shape[0]
    rho = mass * cubic_kernel(np.zeros(n, dtype=pos.dtype), h, 2)
    if pairs.shape[0] == 0:
        return rho
    i, j = pairs[:, 0], pairs[:, 1]
    r = np.sqrt(((pos[i] - pos[j]) ** 2).sum(1))
    w = cubic_kernel(r.astype(pos.dtype), h, 2)
    np.add.at(rho, i, mass[j] * w)
    np.add.at(rho, j, mass[i] * w)
    return rho.astype(T)
