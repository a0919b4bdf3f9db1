"""3-D cubic spline and lattice constants (``tensorsph.threed.kernel3``).

Elementwise helpers used for case set-up (lattice calibration); the pair pass
evaluates the same kernel inside the CUDA gather loops (``csrc/sphkernels.cuh``).
"""
from __future__ import annotations

from functools import lru_cache
import math

import torch

SUPPORT_FACTOR = 2.0


def sigma3(h: float) -> float:
    return 1.0 / (math.pi * h * h * h)


def _shape(q):
    first = 1.0 - 1.5 * q.square() + 0.75 * q.pow(3)
    second = 0.25 * (2.0 - q).clamp_min(0.0).pow(3)
    return torch.where(q < 1.0, first, torch.where(q < 2.0, second, 0.0))


def _shape_prime(q):
    return torch.where(q < 1.0, -3.0 * q + 2.25 * q.square(),
                       torch.where(q < 2.0, -0.75 * (2.0 - q).square(), 0.0))


def _shape_second(q):
    return torch.where(q < 1.0, -3.0 + 4.5 * q, torch.where(q < 2.0, 1.5 * (2.0 - q), 0.0))


def cubic_spline_kernel(r: torch.Tensor, h: float) -> torch.Tensor:
    return sigma3(h) * _shape(r / h).clamp_min(0.0)


def cubic_spline_gradient(delta: torch.Tensor, h: float, eps: float = 1.0e-12) -> torch.Tensor:
    r = torch.linalg.vector_norm(delta, dim=-1)
    return delta * (sigma3(h) * _shape_prime(r / h) / (h * r.clamp_min(eps))).unsqueeze(-1)


def cubic_spline_laplacian(delta: torch.Tensor, h: float, eps: float = 1.0e-12) -> torch.Tensor:
    r = torch.linalg.vector_norm(delta, dim=-1)
    q = r / h
    twice = torch.where(q > 1.0e-10, 2.0 * _shape_prime(q) / q.clamp_min(eps),
                        torch.full_like(q, -6.0))
    radial = _shape_second(q) + twice
    return torch.where(q < 2.0, sigma3(h) * radial / (h * h), torch.zeros_like(radial))


def pair_kernels(delta: torch.Tensor, h: float, eps: float = 1.0e-12):
    r = torch.linalg.vector_norm(delta, dim=-1)
    return (cubic_spline_kernel(r, h), cubic_spline_gradient(delta, h, eps),
            cubic_spline_laplacian(delta, h, eps))


@lru_cache(maxsize=128)
def _lattice_sum(dx: float, h: float, half_width: int) -> float:
    n = torch.arange(-half_width, half_width + 1, dtype=torch.float64) * dx
    grid = torch.cartesian_prod(n, n, n)
    r = torch.linalg.vector_norm(grid, dim=1)
    return float(cubic_spline_kernel(r, h).sum() * dx ** 3)


def lattice_kernel_sum(dx: float, h: float, half_width: int | None = None) -> float:
    if half_width is None:
        half_width = int(math.ceil(SUPPORT_FACTOR * h / dx)) + 1
    return _lattice_sum(float(dx), float(h), int(half_width))


def lattice_bias(dx: float, h: float, half_width: int | None = None) -> float:
    return lattice_kernel_sum(dx, h, half_width) - 1.0


def calibrated_particle_mass(dx: float, h: float, rho0: float, half_width: int | None = None) -> float:
    return rho0 * dx ** 3 / lattice_kernel_sum(dx, h, half_width)
