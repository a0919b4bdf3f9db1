"""Transport-velocity correction on the GPU
(``tensorsph.transport_velocity_correction``).

Keeps the reference API (transport_velocity_correction.py:140-513):
``TVCResult``, the ``no_limiter`` / ``truncated_linear`` limiters,
``kernel_gradient_integral`` and ``transport_velocity_correction``.  The
weighted grad-1 integral of every fluid particle,

    g_i = -[sum_j (C_i + C_j) V_j grad_i W_ij + 2 C_i sum_wall V_j grad_i W_ij],

runs as one gather kernel over symmetric pair rows (``csrc/tvc.cu``), with
the cubic spline normalised in the cloud's dimension and, with ``h_ratio``,
at each particle's own smoothing length ``h_ref / h_ratio``; the displacement
``alpha h_ref^2 limiter(h_ref^2 |g|^2) g`` with its scope, mask and clip runs
as a second kernel.  A limiter other than the two shipped ones is evaluated
by calling it on the device tensor of ``h_ref^2 |g|^2``.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Callable

import torch

from . import _lib
from .droplet_impact import symmetric_rows

__all__ = [
    "TVCResult",
    "kernel_gradient_integral",
    "no_limiter",
    "truncated_linear",
    "transport_velocity_correction",
    "cubic_spline_gradient_dim",
    "SPHINXSYS_DEFAULT_COEFFICIENT",
    "SPHINXSYS_SINGLE_STEP_FRACTION",
    "TRUNCATED_LINEAR_DEFAULT_SLOPE",
    "CUBIC_SPLINE_SIGMA",
]

SPHINXSYS_DEFAULT_COEFFICIENT = 0.2
SPHINXSYS_SINGLE_STEP_FRACTION = 0.25
TRUNCATED_LINEAR_DEFAULT_SLOPE = 100.0

CUBIC_SPLINE_SIGMA: dict[int, Callable[[float], float]] = {
    1: lambda h: 2.0 / (3.0 * h),
    2: lambda h: 10.0 / (7.0 * math.pi * h * h),
    3: lambda h: 1.0 / (math.pi * h * h * h),
}


@dataclass
class TVCResult:
    """Diagnostics of one TVC application."""

    gradient_integral: torch.Tensor
    shift: torch.Tensor
    squared_norm: torch.Tensor
    limiter: torch.Tensor
    alpha: float
    h_ref: float
    clipped: float = 0.0
    extras: dict = field(default_factory=dict)

    @property
    def max_shift(self) -> float:
        if self.shift.numel() == 0:
            return 0.0
        return float(torch.linalg.vector_norm(self.shift, dim=-1).max())

    @property
    def mean_shift(self) -> float:
        if self.shift.numel() == 0:
            return 0.0
        return float(torch.linalg.vector_norm(self.shift, dim=-1).mean())

    @property
    def max_gradient_integral(self) -> float:
        if self.gradient_integral.numel() == 0:
            return 0.0
        return float(torch.linalg.vector_norm(self.gradient_integral, dim=-1).max())


def no_limiter(squared_norm: torch.Tensor) -> torch.Tensor:
    """No damping: the correction is applied in full."""
    return torch.ones_like(squared_norm)


def truncated_linear(slope: float = TRUNCATED_LINEAR_DEFAULT_SLOPE) -> Callable[[torch.Tensor], torch.Tensor]:
    """``min(slope * h_ref^2 |g|^2, 1)``: attenuates the correction where the
    grad-1 inconsistency is small.  A finite positive slope is required."""
    if not math.isfinite(slope) or slope <= 0.0:
        raise ValueError("TruncatedLinear slope must be finite and positive")

    def limiter(squared_norm: torch.Tensor) -> torch.Tensor:
        return torch.minimum(slope * squared_norm, torch.ones_like(squared_norm))

    limiter.__name__ = f"truncated_linear({slope:g})"
    limiter.truncated_linear_slope = float(slope)
    return limiter


def cubic_spline_gradient_dim(delta: torch.Tensor, h, dim: int, eps: float = 1.0e-12) -> torch.Tensor:
    """``grad_i W_ij`` of the cubic spline in ``dim`` dimensions (per-pair
    helper; the corrections themselves run on the device kernels)."""
    if dim not in CUBIC_SPLINE_SIGMA:
        raise ValueError(f"cubic spline is implemented for dim in 1..3, got {dim}")
    r = torch.linalg.vector_norm(delta, dim=-1)
    q = r / h
    sigma = CUBIC_SPLINE_SIGMA[dim](h) if not torch.is_tensor(h) else {
        1: 2.0 / (3.0 * h), 2: 10.0 / (7.0 * math.pi * h * h), 3: 1.0 / (math.pi * h * h * h)}[dim]
    dshape = torch.where(q < 1.0, -3.0 * q + 2.25 * q.square(),
                         torch.where(q < 2.0, -0.75 * (2.0 - q).square(), 0.0))
    return delta * (sigma * dshape / (h * r.clamp_min(eps))).unsqueeze(-1)


def _as_ratio(h_ratio, n: int, like: torch.Tensor) -> torch.Tensor:
    if isinstance(h_ratio, torch.Tensor):
        r = h_ratio.to(dtype=like.dtype, device=like.device).reshape(-1)
        if r.numel() == n:
            return r
        if r.numel() < n:
            return torch.cat([r, torch.ones(n - r.numel(), dtype=like.dtype, device=like.device)])
        raise ValueError("h_ratio has more entries than particles")
    return torch.full((n,), float(h_ratio), dtype=like.dtype, device=like.device)


def _checked(positions, volume, h, wall_count, dim):
    n_total = positions.shape[0]
    if volume.shape != (n_total,):
        raise ValueError("volume must have one entry per position")
    if not math.isfinite(h) or h <= 0:
        raise ValueError("h must be finite and positive")
    dim = int(positions.shape[1]) if dim is None else int(dim)
    if dim != int(positions.shape[1]):
        raise ValueError(f"dim={dim} contradicts the point cloud (positions.shape[1]="
                         f"{int(positions.shape[1])})")
    if dim not in CUBIC_SPLINE_SIGMA:
        raise ValueError(f"cubic spline is implemented for dim in 1..3, got {dim}")
    n_fluid = n_total - int(wall_count)
    if n_fluid <= 0:
        raise ValueError("need at least one fluid particle")
    return n_total, n_fluid, dim


def _gradient(positions, volume, h, pairs, ratio, h_scale, wall_count, wall_factor, correction, dim):
    """Device gather of g and |g|^2 (fluid rows); returns device tensors and
    the prepared inputs."""
    n_total, n_fluid, dim = _checked(positions, volume, h, wall_count, dim)
    dev = _lib.cuda_device(positions)
    dtype = positions.dtype
    P = _lib.to_dev(positions.detach(), dev)
    Vol = _lib.to_dev(volume.detach(), dev, dtype)
    if pairs is None:
        from .neighbor_search import cell_linked_pairs
        search_h = h
        if ratio is not None:
            search_h = h / float(_as_ratio(ratio, n_total, positions).min().clamp_min(1.0e-30))
        pairs = cell_linked_pairs(P, 2.0 * search_h)
    rowptr, entries = symmetric_rows(_lib.to_dev(pairs, dev), n_total)
    # the kernel's ratio over all particles (walls padded with 1), fluid rows only
    R = None if ratio is None else _as_ratio(ratio, n_total, P)[:n_fluid].contiguous()
    C = None if correction is None else _lib.to_dev(correction.detach(), dev, dtype)
    grad = torch.empty((n_fluid, dim), dtype=dtype, device=dev)
    squared = torch.empty(n_fluid, dtype=dtype, device=dev)
    prm = _lib.TvcParams()
    prm.n_total, prm.n_fluid, prm.dim, prm.dtype = n_total, n_fluid, dim, _lib.dtype_code(dtype)
    prm.has_ratio = int(R is not None)
    prm.h, prm.h_ratio_scale, prm.wall_factor = float(h), float(h_scale), float(wall_factor)
    io = _lib.TvcIO()
    io.pos, io.volume, io.rowptr, io.entries = P.data_ptr(), Vol.data_ptr(), rowptr.data_ptr(), entries.data_ptr()
    io.h_ratio = 0 if R is None else R.data_ptr()
    io.correction = 0 if C is None else C.data_ptr()
    io.gradient, io.squared = grad.data_ptr(), squared.data_ptr()
    _lib.check(_lib.lib().tsph_tvc_gradient(ctypes.byref(prm), ctypes.byref(io), _lib.stream(dev)),
               "tsph_tvc_gradient")
    return prm, io, grad, squared, R, (rowptr, entries, P, Vol, C)


def kernel_gradient_integral(positions: torch.Tensor, volume: torch.Tensor, h: float,
                             pairs: torch.Tensor | None = None, h_ratio: float | torch.Tensor | None = None,
                             wall_count: int = 0, wall_factor: float = 2.0,
                             correction: torch.Tensor | None = None, dim: int | None = None) -> torch.Tensor:
    """The (negated, weighted) grad-1 integral of the fluid particles, ``(N, D)``."""
    out_device = positions.device
    _, _, grad, _, _, _ = _gradient(positions, volume, h, pairs, h_ratio, 1.0, wall_count, wall_factor,
                                    correction, dim)
    return grad.to(out_device)


def transport_velocity_correction(positions: torch.Tensor, volume: torch.Tensor, h: float,
                                  alpha: float | None = None, pairs: torch.Tensor | None = None,
                                  h_ratio: float | torch.Tensor | None = None, wall_count: int = 0,
                                  h_ref: float | None = None,
                                  limiter: Callable[[torch.Tensor], torch.Tensor] | None = None,
                                  max_shift: float | None = None, active: torch.Tensor | None = None,
                                  scope_tol: float | None = None, dim: int | None = None) -> TVCResult:
    """One correction ``delta r_i = alpha h_ref^2 limiter(h_ref^2 |g_i|^2) g_i``
    (``alpha=None``: the single-acoustic-step default 0.2 / 4)."""
    if alpha is None:
        alpha = SPHINXSYS_DEFAULT_COEFFICIENT * SPHINXSYS_SINGLE_STEP_FRACTION
    if h_ref is None:
        h_ref = h
    if limiter is None:
        limiter = no_limiter
    if scope_tol is not None and (not math.isfinite(scope_tol) or scope_tol < 0.0):
        raise ValueError("scope_tol must be finite and non-negative")
    out_device = positions.device
    prm, io, grad, squared, R, keep = _gradient(positions, volume, h, pairs, h_ratio, h / h_ref, wall_count,
                                                2.0, None, dim)
    n_fluid, dev, dtype = int(prm.n_fluid), grad.device, grad.dtype
    if active is not None and tuple(active.shape) != (n_fluid,):
        raise ValueError("active must be (N,) over the fluid particles")
    given = None
    if limiter is no_limiter:
        prm.limiter = 0
    elif getattr(limiter, "truncated_linear_slope", None) is not None:
        prm.limiter, prm.slope = 1, limiter.truncated_linear_slope
    else:
        prm.limiter = 2
        given = limiter(h_ref * h_ref * squared).to(dtype=dtype, device=dev).contiguous()
    A = None if active is None else active.to(device=dev, dtype=torch.uint8).contiguous()
    prm.alpha, prm.h_ref = float(alpha), float(h_ref)
    prm.has_scope_tol, prm.scope_tol = int(scope_tol is not None), float(scope_tol or 0.0)
    prm.has_max_shift, prm.max_shift = int(max_shift is not None), float(max_shift or 0.0)
    if h_ratio is not None:
        # the displacement divides by the unscaled ratio of the fluid particles
        R = _as_ratio(h_ratio, n_fluid, grad).contiguous()
        io.h_ratio = R.data_ptr()
    fac = torch.empty(n_fluid, dtype=dtype, device=dev)
    shift = torch.empty_like(grad)
    clipped = torch.zeros(1, dtype=torch.int64, device=dev)
    io.limiter_in = 0 if given is None else given.data_ptr()
    io.active = 0 if A is None else A.data_ptr()
    io.limiter_out, io.shift, io.clipped = fac.data_ptr(), shift.data_ptr(), clipped.data_ptr()
    _lib.check(_lib.lib().tsph_tvc_shift(ctypes.byref(prm), ctypes.byref(io), _lib.stream(dev)), "tsph_tvc_shift")
    n_clip = int(clipped.item())
    ratio_range = None
    if h_ratio is not None:
        ratio_range = (float(min(R.min().cpu(), torch.tensor(float("inf")))), float(R.max()))
    return TVCResult(
        gradient_integral=grad.to(out_device), shift=shift.to(out_device), squared_norm=squared.to(out_device),
        limiter=fac.to(out_device), alpha=float(alpha), h_ref=float(h_ref),
        clipped=(n_clip / n_fluid if max_shift is not None and n_fluid else 0.0),
        extras={"max_shift": max_shift, "h_ratio": ratio_range,
                "dim": int(prm.dim), "scope_tol": scope_tol,
                "scope_tol_kept_fraction": (None if scope_tol is None else float(
                    ((torch.linalg.vector_norm(grad, dim=1) * h_ref) <= scope_tol).to(dtype).mean())),
                "scope_active_fraction": (1.0 if active is None else float(A.to(dtype).mean()))})
