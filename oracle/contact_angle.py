"""Oracle (test infrastructure only): the wall contact-angle terms of the 2-D
CSF, in numpy, in the dtype of the positions.

* ``nearest_wall``     csf_consistent.py:449-480: distance to the nearest
  wall particle (first of equals) and the unit direction from it to the
  particle; a particle sitting on a wall particle takes the mean direction of
  the others.  Distances are exact here; the reference's ``torch.cdist`` forms
  them from dot products, which only matters for exact ties.
* ``apply_contact_angle_boundary``  csf_consistent.py:483-560: within
  ``reach h`` of the wall the normal ``-grad c / |grad c|`` is blended
  linearly (full at the wall) toward ``cos(theta) n_wall + sin(theta) t`` and
  ``|grad c|`` is kept.
* ``wall_spacing``, ``wall_delta``, ``wall_adhesion_force``
  contact_angle_isph.py:75-213: the wall surface delta ``sum_k W A / (1/2)``
  with ``A`` the squared median nearest-neighbour wall spacing, the weight
  ``clip(delta_w / 0.4734, 0, 1)`` and the traction ``C sigma delta_s w d``,
  ``d = cos(theta) t_wall`` ("young") or ``n_wall - cos(theta) n``
  ("brackbill").

Pinned to ``tests/golden/contact.npz``.
"""
from __future__ import annotations

import math

import numpy as np

from .pairpass import cubic_kernel

DEFAULT_WALL_DELTA_REF = 0.4734
DEFAULT_TRACTION_CALIBRATION = 0.9611


def nearest_wall(pos, wall):
    T = pos.dtype.type
    d2 = ((pos[:, None, :] - wall[None, :, :]) ** 2).sum(-1)
    idx = d2.argmin(axis=1)
    dmin = np.sqrt(d2[np.arange(pos.shape[0]), idx])
    normal = pos - wall[idx]
    mag = np.maximum(np.sqrt((normal * normal).sum(1)), T(1e-30))
    degenerate = mag < T(1e-12)
    if degenerate.any():
        mean = normal[~degenerate].mean(axis=0) if (~degenerate).any() else np.zeros(pos.shape[1], pos.dtype)
        fb = mean / max(np.sqrt((mean * mean).sum()), T(1e-30))
        normal = np.where(degenerate[:, None], fb[None, :], normal)
        mag = np.maximum(np.sqrt((normal * normal).sum(1)), T(1e-30))
    return dmin.astype(pos.dtype), (normal / mag[:, None]).astype(pos.dtype)


def apply_contact_angle_boundary(grad_c, pos, wall, h, theta, reach=2.0):
    T = pos.dtype.type
    out = grad_c.copy()
    if wall is None or wall.size == 0 or grad_c.size == 0:
        return out
    d, n_wall = nearest_wall(pos, wall)
    mag = np.sqrt((grad_c * grad_c).sum(1))
    active = (d < T(reach * h)) & (mag > 0)
    if not active.any():
        return out
    n = -grad_c[active] / mag[active][:, None]
    wn = n_wall[active]
    tangent = n - (n * wn).sum(1, keepdims=True) * wn
    perp = np.stack([-wn[:, 1], wn[:, 0]], 1)
    sgn = np.where((tangent * perp).sum(1, keepdims=True) < 0, T(-1), T(1))
    tangent = perp * sgn
    target = T(math.cos(theta)) * wn + T(math.sin(theta)) * tangent
    blend = np.clip(T(1) - d[active] / T(reach * h), T(0), T(1))[:, None]
    mixed = (T(1) - blend) * n + blend * target
    mixed = mixed / np.maximum(np.sqrt((mixed * mixed).sum(1, keepdims=True)), T(1e-30))
    out[active] = -mag[active][:, None] * mixed
    return out.astype(pos.dtype)


def wall_spacing(wall):
    if wall.shape[0] < 2:
        return 1.0
    d = np.sqrt(((wall[:, None, :] - wall[None, :, :]) ** 2).sum(-1))
    np.fill_diagonal(d, np.inf)
    nn = np.sort(d.min(axis=1))
    return float(nn[(nn.size - 1) // 2])      # lower median, as torch.median


def wall_delta(pos, wall, h):
    T = pos.dtype.type
    area = wall_spacing(wall) ** pos.shape[1]
    d = np.sqrt(((pos[:, None, :] - wall[None, :, :]) ** 2).sum(-1))
    return (cubic_kernel(d, h, 2).sum(axis=1) * T(area / 0.5)).astype(pos.dtype)


def wall_adhesion_force(pos, wall, normal, theta, sigma, delta_s, h, calibration=DEFAULT_TRACTION_CALIBRATION,
                        model="young"):
    T = pos.dtype.type
    w = np.clip(wall_delta(pos, wall, h) / T(DEFAULT_WALL_DELTA_REF), T(0), T(1))
    _, n_wall = nearest_wall(pos, wall)
    cos_t = math.cos(theta)
    if model == "young":
        tangent = normal - (normal * n_wall).sum(1, keepdims=True) * n_wall
        mag = np.sqrt((tangent * tangent).sum(1, keepdims=True))
        fb = np.zeros_like(tangent)
        fb[:, 0] = 1
        fb = fb - (fb * n_wall).sum(1, keepdims=True) * n_wall
        fb = fb / np.maximum(np.sqrt((fb * fb).sum(1, keepdims=True)), T(1e-30))
        direction = np.where(mag < T(1e-9), fb, tangent / np.maximum(mag, T(1e-30))) * T(cos_t)
    elif model == "brackbill":
        direction = n_wall - T(cos_t) * normal
    else:
        raise ValueError(f"unknown contact-angle force model {model!r}")
    coef = T(calibration * sigma) * delta_s * w
    return (coef[:, None] * direction).astype(pos.dtype)
