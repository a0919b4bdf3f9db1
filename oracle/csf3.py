"""Oracle: the 3-D CSF surface tension (threed/csf3.py) in numpy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, with the reference's pair-list scatter structure (``np.add.at`` for
``index_add``) and in the dtype of the positions:

* ``_mls_matrix``                     src/tensorsph/threed/csf3.py:98-112
* ``csf_fields3`` ("mls" curvature)   src/tensorsph/threed/csf3.py:115-165
* ``curvature_axisymmetric``          src/tensorsph/threed/csf3.py:168-220: the
  2-D quadratic interface fit (``oracle.csf.fit_curvature_quadratic``, 4h
  stencil, zero fallback) on the meridional projection (r, z) of the particles
  and of their normals, plus n_r / max(r, h / 4)
* ``surface_tension_acceleration3``   src/tensorsph/threed/csf3.py:220-238
* pair geometry (minimum image)       src/tensorsph/threed/operators3.py:51-67
* 3-D cubic spline and its gradient   src/tensorsph/threed/kernel3.py:90-105

Pinned to ``tests/golden/csf3.npz`` and ``tests/golden/csf3axi.npz`` (written
by running the reference).
"""
from __future__ import annotations

import numpy as np

from .neighbors import minimum_image
from .pairpass import cubic_kernel, cubic_pair_kernels

__all__ = ["csf_fields3", "curvature_axisymmetric", "surface_tension_acceleration3"]


def _lower_median(x):
    """torch.median of a flat tensor: the lower of the two middle values."""
    s = np.sort(x)
    return s[(s.size - 1) // 2]


def curvature_axisymmetric(pos, normal, delta_s, pairs, h):
    """Curvature of a surface of revolution about z: meridional fit + n_r / r."""
    from .csf import fit_curvature_quadratic
    dt = pos.dtype.type
    r = np.sqrt(pos[:, 0] * pos[:, 0] + pos[:, 1] * pos[:, 1])
    mer = np.stack((r, pos[:, 2]), axis=1)
    radial = pos[:, :2] / np.maximum(r, dt(1e-30))[:, None]
    n_r = (normal[:, :2] * radial).sum(axis=1)
    m = np.stack((n_r, normal[:, 2]), axis=1)
    m_normal = m / np.maximum(np.sqrt((m * m).sum(axis=1)), dt(1e-30))[:, None]
    k_mer = fit_curvature_quadratic(mer, m_normal, delta_s, pairs, h, np.zeros_like(r))
    return (k_mer + n_r / np.maximum(r, dt(0.25 * h))).astype(pos.dtype)


def csf_fields3(pos, mass, h, pairs, *, rho0, box=None, volume=None, curvature="mls"):
    """``dict(color, grad_c, normal, kappa, delta_s, valid)`` of a 3-D cloud."""
    dt = pos.dtype.type
    n, dim = pos.shape
    vol = mass / dt(rho0) if volume is None else volume
    i, j = pairs[:, 0], pairs[:, 1]
    delta = pos[i] - pos[j]
    if box is not None:
        delta = minimum_image(delta, np.asarray(box, dtype=pos.dtype))
    weight, grad = cubic_pair_kernels(delta, h, 3)
    self_weight = cubic_kernel(np.zeros(1, dtype=pos.dtype), h, 3)[0]

    color = np.zeros(n, dtype=pos.dtype)
    np.add.at(color, i, vol[j] * weight)
    np.add.at(color, j, vol[i] * weight)
    color = color + vol * self_weight

    # M_i = sum_j V_j (x_j - x_i) (x) grad_i W_ij, the same term for both ends
    outer = -np.einsum("pa,pb->pab", delta, grad)
    big_m = np.zeros((n, dim, dim), dtype=pos.dtype)
    np.add.at(big_m, i, vol[j, None, None] * outer)
    np.add.at(big_m, j, vol[i, None, None] * outer)
    det = np.linalg.det(big_m)
    scale = max(_lower_median(np.abs(det)), dt(1e-30))
    valid = np.abs(det) > dt(1e-6) * scale
    big_m = np.where(valid[:, None, None], big_m, np.eye(dim, dtype=pos.dtype))

    dc = color[j] - color[i]
    num = np.zeros((n, dim), dtype=pos.dtype)
    np.add.at(num, i, (vol[j] * dc)[:, None] * grad)
    np.add.at(num, j, (vol[i] * dc)[:, None] * grad)
    grad_c = np.linalg.solve(big_m, num[..., None])[..., 0]

    delta_s = np.sqrt((grad_c * grad_c).sum(axis=1))
    normal = -grad_c / np.maximum(delta_s, dt(1e-30))[:, None]

    dn = normal[j] - normal[i]
    outer_n = np.einsum("pa,pb->pab", dn, grad)
    s_mat = np.zeros((n, dim, dim), dtype=pos.dtype)
    np.add.at(s_mat, i, vol[j, None, None] * outer_n)
    np.add.at(s_mat, j, vol[i, None, None] * outer_n)
    inv = np.linalg.inv(big_m)
    kappa = (s_mat * np.transpose(inv, (0, 2, 1))).sum(axis=(1, 2))
    kappa = np.where(valid, kappa, dt(0))
    if curvature == "axisym":
        kappa = curvature_axisymmetric(pos, normal, delta_s, pairs, h)
    elif curvature != "mls":
        raise ValueError(f"unknown curvature {curvature!r}")
    return dict(color=color, grad_c=grad_c, normal=normal, kappa=kappa, delta_s=delta_s, valid=valid)


def surface_tension_acceleration3(state, rho, sigma, cutoff=1.0e-3):
    """``a = -sigma kappa delta_s n / rho`` on particles with
    ``delta_s > cutoff * max(delta_s)``."""
    normal = state["normal"]
    if sigma == 0.0:
        return np.zeros_like(normal)
    dt = normal.dtype.type
    weight = state["delta_s"]
    limit = dt(cutoff) * weight.max() if weight.size else dt(0)
    active = (weight > limit).astype(weight.dtype)
    scale = -(dt(sigma) * state["kappa"] * weight * active / rho)
    return scale[:, None] * normal
