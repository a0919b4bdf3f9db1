"""Oracle: transport-velocity correction in numpy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, with the reference's pair scatter structure and in the dtype of
the positions:

* ``truncated_linear``                 src/tensorsph/transport_velocity_correction.py:180-223
* ``cubic_spline_gradient_dim``        src/tensorsph/transport_velocity_correction.py:261-282
* ``kernel_gradient_integral``         src/tensorsph/transport_velocity_correction.py:285-410
* ``transport_velocity_correction``    src/tensorsph/transport_velocity_correction.py:413-513

Pinned to ``tests/golden/tvc.npz`` (written by running the reference).
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["kernel_gradient_integral", "transport_velocity_correction"]

_SIGMA = {1: lambda h: 2.0 / (3.0 * h), 2: lambda h: 10.0 / (7.0 * math.pi * h * h),
          3: lambda h: 1.0 / (math.pi * h * h * h)}


def _gradient(delta, h, dim, eps=1.0e-12):
    """grad_i W_ij of the cubic spline in ``dim`` dimensions; ``h`` a scalar
    or one value per pair."""
    dt = delta.dtype.type
    h = np.asarray(h, dtype=delta.dtype)
    r = np.sqrt((delta * delta).sum(axis=-1))
    q = r / h
    sigma = (np.asarray(_SIGMA[dim](1.0), dtype=delta.dtype) / h ** dim if dim != 2
             else np.asarray(10.0 / (7.0 * math.pi), dtype=delta.dtype) / (h * h))
    dshape = np.where(q < 1.0, -3.0 * q + 2.25 * q * q,
                      np.where(q < 2.0, -0.75 * (2.0 - q) ** 2, 0.0)).astype(delta.dtype)
    scale = sigma * dshape / (h * np.maximum(r, dt(eps)))
    return delta * scale[..., None]


def kernel_gradient_integral(positions, volume, h, pairs, h_ratio=None, wall_count=0, wall_factor=2.0,
                             correction=None):
    """``-[sum_j (C_i + C_j) grad_i W_ij V_j + wall_factor C_i sum_wall grad_i W_ij V_j]``
    (C = 1 unless given) for the fluid particles (the first ``n - wall_count``)."""
    n_total, dim = positions.shape
    n_fluid = n_total - int(wall_count)
    grad = np.zeros((n_fluid, dim), dtype=positions.dtype)
    if pairs.shape[0] == 0:
        return grad
    i, j = pairs[:, 0], pairs[:, 1]
    delta = positions[i] - positions[j]
    if h_ratio is None:
        gw_i = _gradient(delta, h, dim)
        gw_j = -gw_i
    else:
        ratio = np.ones(n_total, dtype=positions.dtype)
        ratio[:np.asarray(h_ratio).size] = h_ratio
        h_local = positions.dtype.type(h) / ratio
        gw_i = _gradient(delta, h_local[i], dim)
        gw_j = _gradient(-delta, h_local[j], dim)
    c = np.ones(n_total, dtype=positions.dtype) if correction is None else correction
    fi, fj = i < n_fluid, j < n_fluid
    ff, fw, wf = fi & fj, fi & ~fj, ~fi & fj
    dt = positions.dtype.type
    np.add.at(grad, i[ff], ((c[i[ff]] + c[j[ff]]) * volume[j[ff]])[:, None] * gw_i[ff])
    np.add.at(grad, j[ff], ((c[i[ff]] + c[j[ff]]) * volume[i[ff]])[:, None] * gw_j[ff])
    np.add.at(grad, i[fw], (dt(wall_factor) * c[i[fw]] * volume[j[fw]])[:, None] * gw_i[fw])
    np.add.at(grad, j[wf], (dt(wall_factor) * c[j[wf]] * volume[i[wf]])[:, None] * gw_j[wf])
    return -grad


def transport_velocity_correction(positions, volume, h, pairs, *, alpha=None, h_ratio=None, wall_count=0,
                                  h_ref=None, slope=None, max_shift=None, active=None, scope_tol=None):
    """``dict(gradient_integral, shift, squared_norm, limiter, clipped)``;
    ``slope`` selects TruncatedLinear (None: no limiter)."""
    dt = positions.dtype.type
    alpha = 0.2 * 0.25 if alpha is None else alpha
    h_ref = h if h_ref is None else h_ref
    ratio = None
    if h_ratio is not None:
        ratio = np.asarray(h_ratio, dtype=positions.dtype) * dt(h / h_ref)
    g = kernel_gradient_integral(positions, volume, h, pairs, h_ratio=ratio, wall_count=wall_count)
    squared = (g * g).sum(axis=1)
    measure = dt(h_ref * h_ref) * squared
    fac = np.ones_like(squared) if slope is None else np.minimum(dt(slope) * measure, dt(1))
    shift = dt(alpha * h_ref * h_ref) * fac[:, None] * g
    if h_ratio is not None:
        inv = dt(1) / np.asarray(h_ratio, dtype=positions.dtype)
        shift = shift * (inv * inv)[:, None]
    if active is not None:
        shift = shift * np.asarray(active)[:, None].astype(shift.dtype)
    if scope_tol is not None:
        keep = np.sqrt((g * g).sum(axis=1)) * dt(h_ref) <= dt(scope_tol)
        shift = shift * keep[:, None].astype(shift.dtype)
    clipped = 0.0
    if max_shift is not None:
        norm = np.sqrt((shift * shift).sum(axis=1))
        over = norm > max_shift
        clipped = float(over.mean()) if norm.size else 0.0
        scale = np.where(over, dt(max_shift) / np.maximum(norm, dt(1e-30)), dt(1))
        shift = shift * scale[:, None]
    return dict(gradient_integral=g, shift=shift, squared_norm=squared, limiter=fac, clipped=clipped)
