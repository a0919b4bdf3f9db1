"""Oracle (test infrastructure only): CSF surface tension, consistent scheme.

numpy restatement of the 2-D surface-tension path the droplet case runs
(``Config.csf_scheme = "consistent"``, ``csf_curvature = "fit_quadratic"``,
``csf_delta_normalization = "legacy"``):

* colour  c_i = V_i W(0) + sum_j V_j W_ij, V = m / rho0, clipped to [0, 1]
  (csf_consistent.py:177-201);
* MLS matrix M_i = sum_j V_j (x_j - x_i) (x) grad_i W_ij, replaced by the
  identity where |det M| <= 1e-4 median|det M| (csf_consistent.py:85-114);
* grad c = M^-T sum_j V_j (c_j - c_i) grad_i W_ij (:117-137); outward normal
  -grad c / |grad c| where |grad c| > 1e-12, two Shepard passes (self term in
  the denominator only, :204-230) renormalised on the interface (:320-330);
* kappa_mls = trace(S M^-1), S = sum_j V_j (n_j - n_i) (x) grad_i W_ij
  (:140-160); delta_s = 2 |grad c| (:368-370);
* curvature: weighted quadratic fit v = c + b u + a u^2 in the frame (t, n)
  of each particle over the 4h stencil, weights w_j = clamp(delta_s_j /
  max delta_s), kappa = -2a / (1 + b^2)^1.5 where the particle is active
  (w > 0.05) and the 3x3 system is regular (|det| > 1e-6 max|det|), else
  kappa_mls (csf_curvature.py:78-166); or the Pratt circle fit with the same
  weights (``curvature_scheme="fit_circle"``, :179-213);
* a = -sigma kappa delta_s n / rho with delta_s = 0 where |grad c| <= 1e-3 max
  (csf_consistent.py:384-446).  All pairs are the 4h list, as the reference
  builds it for the fit (:415-421).

The variants of ``csf_fields`` (csf_consistent.py:262-381) are restated as
well: ``curvature_scheme="mls"`` (no fit), ``delta_normalization=
"local_range"`` (|grad c| over the local colour range max - min of the pair
neighbourhood, clipped to [0.2, 1]; :231-259), ``normal_smoothing`` passes
and ``curvature_color_smoothing`` (the curvature from a Shepard-smoothed,
clipped colour field while the force keeps the sharp one).  Pinned to
``tests/golden/csf.npz`` and ``tests/golden/csf2d.npz``.
"""
from __future__ import annotations

import numpy as np

from .neighbors import cell_linked_pairs
from .pairpass import cubic_kernel, cubic_pair_kernels


def _pair_geometry(pos, pairs, h):
    i, j = pairs[:, 0], pairs[:, 1]
    delta = pos[i] - pos[j]
    w, gw = cubic_pair_kernels(delta, h, 2)
    return i, j, delta, w, gw


def colour(pos, vol, pairs, h):
    T = pos.dtype.type
    c = vol * cubic_kernel(np.zeros(pos.shape[0], dtype=pos.dtype), h, 2)
    i, j, _, w, _ = _pair_geometry(pos, pairs, h)
    np.add.at(c, i, vol[j] * w)
    np.add.at(c, j, vol[i] * w)
    return np.clip(c, T(0), T(1))


def mls_matrix(pos, vol, pairs, h):
    n = pos.shape[0]
    i, j, delta, _, gw = _pair_geometry(pos, pairs, h)
    outer = -np.einsum("pa,pb->pab", delta, gw)
    m = np.zeros((n, 2, 2), dtype=pos.dtype)
    np.add.at(m, i, vol[j, None, None] * outer)
    np.add.at(m, j, vol[i, None, None] * outer)
    det = m[:, 0, 0] * m[:, 1, 1] - m[:, 0, 1] * m[:, 1, 0]
    # torch.median returns the lower of the two middle values
    med = np.sort(np.abs(det))[(n - 1) // 2]
    scale = max(med, pos.dtype.type(1e-30))
    ok = np.abs(det) > 1e-4 * scale
    m[~ok] = np.eye(2, dtype=pos.dtype)
    return m, ok


def mls_gradient(pos, field, vol, pairs, h, m):
    n = pos.shape[0]
    i, j, _, _, gw = _pair_geometry(pos, pairs, h)
    df = field[j] - field[i]
    contrib = df[:, None] * gw
    rhs = np.zeros((n, 2), dtype=pos.dtype)
    np.add.at(rhs, i, vol[j, None] * contrib)
    np.add.at(rhs, j, vol[i, None] * contrib)
    return np.linalg.solve(np.transpose(m, (0, 2, 1)), rhs[..., None])[..., 0]


def mls_divergence(pos, field, vol, pairs, h, m):
    n = pos.shape[0]
    i, j, _, _, gw = _pair_geometry(pos, pairs, h)
    df = field[j] - field[i]
    contrib = np.einsum("pa,pb->pab", df, gw)
    s = np.zeros((n, 2, 2), dtype=pos.dtype)
    np.add.at(s, i, vol[j, None, None] * contrib)
    np.add.at(s, j, vol[i, None, None] * contrib)
    inv = np.linalg.inv(m)
    return (s * np.transpose(inv, (0, 2, 1))).sum(axis=(1, 2))


def shepard_smooth(field, pos, vol, pairs, h, passes):
    i, j, _, w, _ = _pair_geometry(pos, pairs, h)
    out = field
    w0 = cubic_kernel(np.zeros(1, dtype=pos.dtype), h, 2)[0]
    for _ in range(passes):
        num = np.zeros_like(out)
        den = vol * w0
        np.add.at(num, i, (vol[j] * w)[:, None] * out[j])
        np.add.at(den, i, vol[j] * w)
        np.add.at(num, j, (vol[i] * w)[:, None] * out[i])
        np.add.at(den, j, vol[i] * w)
        out = num / np.maximum(den, pos.dtype.type(1e-30))[:, None]
    return out


def fit_curvature_quadratic(pos, normal, delta_s, pairs, h, fallback, stencil=4.0,
                            min_weight_fraction=0.05):
    T = pos.dtype.type
    n = pos.shape[0]
    ds_max = max(delta_s.max(), T(1e-30))
    w_node = np.clip(delta_s / ds_max, T(0), T(1))
    i, j = pairs[:, 0], pairs[:, 1]
    delta = pos[i] - pos[j]
    r = np.sqrt((delta * delta).sum(1))
    inside = r <= T(stencil * h)
    w_ij = np.where(inside, w_node[j], T(0))
    w_ji = np.where(inside, w_node[i], T(0))
    active = w_node > min_weight_fraction
    tangent = np.stack([-normal[:, 1], normal[:, 0]], axis=1)
    u_i = (-delta * tangent[i]).sum(1)
    v_i = (-delta * normal[i]).sum(1)
    u_j = (delta * tangent[j]).sum(1)
    v_j = (delta * normal[j]).sum(1)

    def moments(u, v, w, dst):
        feats = np.stack([np.ones_like(u), u, v, u * u, u * v, u * u * u, u * u * v, u * u * u * u]) * w
        out = np.zeros((8, n), dtype=pos.dtype)
        for k in range(8):
            np.add.at(out[k], dst, feats[k])
        return out

    s = moments(u_i, v_i, w_ij, i) + moments(u_j, v_j, w_ji, j)
    s[0] = s[0] + w_node
    s0, s1, s2, s3, s4, s5, s6, s7 = s
    mat = np.zeros((n, 3, 3), dtype=pos.dtype)
    mat[:, 0] = np.stack([s0, s1, s3], 1)
    mat[:, 1] = np.stack([s1, s3, s5], 1)
    mat[:, 2] = np.stack([s3, s5, s7], 1)
    rhs = np.stack([s2, s4, s6], 1)
    det = np.linalg.det(mat)
    scale = max(np.abs(det).max(), T(1e-30))
    ok = active & (np.abs(det) > T(1e-6) * scale)
    mat[~ok] = np.eye(3, dtype=pos.dtype)
    sol = np.linalg.solve(mat, rhs[..., None])[..., 0]
    b, a = sol[:, 1], sol[:, 2]
    kappa = -2.0 * a / (1.0 + b * b) ** 1.5
    return np.where(ok, kappa, fallback).astype(pos.dtype)


def fit_curvature_circle(pos, normal, delta_s, pairs, h, fallback, stencil=4.0, min_weight_fraction=0.05):
    """Pratt algebraic circle fit x^2 + y^2 + D x + E y + F = 0 in the frame
    centred on each particle, same weights and activity as the quadratic fit;
    kappa = -sign(c . n) / r with c = -(D, E) / 2, r = sqrt(|c|^2 - F), where
    the 3x3 system is regular and c . n != 0 (csf_curvature.py:179-213)."""
    T = pos.dtype.type
    n = pos.shape[0]
    ds_max = max(delta_s.max(), T(1e-30))
    w_node = np.clip(delta_s / ds_max, T(0), T(1))
    i, j = pairs[:, 0], pairs[:, 1]
    delta = pos[i] - pos[j]
    r = np.sqrt((delta * delta).sum(1))
    inside = r <= T(stencil * h)
    w_ij = np.where(inside, w_node[j], T(0))
    w_ji = np.where(inside, w_node[i], T(0))
    active = w_node > min_weight_fraction

    def moments(x, y, w, dst):
        f = x * x + y * y
        feats = np.stack([np.ones_like(x), x, y, x * x, x * y, y * y, x * f, y * f, f]) * w
        out = np.zeros((9, n), dtype=pos.dtype)
        for k in range(9):
            np.add.at(out[k], dst, feats[k])
        return out

    z = moments(-delta[:, 0], -delta[:, 1], w_ij, i) + moments(delta[:, 0], delta[:, 1], w_ji, j)
    z[0] = z[0] + w_node
    mat = np.zeros((n, 3, 3), dtype=pos.dtype)
    mat[:, 0] = np.stack([z[3], z[4], z[1]], 1)
    mat[:, 1] = np.stack([z[4], z[5], z[2]], 1)
    mat[:, 2] = np.stack([z[1], z[2], z[0]], 1)
    rhs = -np.stack([z[6], z[7], z[8]], 1)
    det = np.linalg.det(mat)
    scale = max(np.abs(det).max(), T(1e-30))
    ok = active & (np.abs(det) > T(1e-6) * scale)
    mat[~ok] = np.eye(3, dtype=pos.dtype)
    sol = np.linalg.solve(mat, rhs[..., None])[..., 0]
    cx, cy = T(-0.5) * sol[:, 0], T(-0.5) * sol[:, 1]
    rad = np.sqrt(np.maximum(cx * cx + cy * cy - sol[:, 2], T(1e-30)))
    sign = np.sign(cx * normal[:, 0] + cy * normal[:, 1])
    kappa = -sign / np.maximum(rad, T(1e-30))
    ok = ok & (sign != 0)
    return np.where(ok, kappa, fallback).astype(pos.dtype)


def _normal(pos, field, vol, pairs, h, m, passes, bc=None):
    """Outward normal of a colour field with ``passes`` Shepard passes
    (``bc``: the wall boundary applied to the gradient first)."""
    T = pos.dtype.type
    grad = mls_gradient(pos, field, vol, pairs, h, m)
    if bc is not None:
        grad = bc(grad)
    mag = np.sqrt((grad * grad).sum(1))
    tiny = T(1e-12)
    normal = np.where(mag[:, None] > tiny, -grad / np.maximum(mag, tiny)[:, None], T(0))
    if passes:
        sm = shepard_smooth(normal, pos, vol, pairs, h, passes)
        nrm = np.sqrt((sm * sm).sum(1))
        normal = np.where(mag[:, None] > tiny, sm / np.maximum(nrm, tiny)[:, None], normal)
    return grad, mag, normal


def colour_range(color, pairs):
    """max - min of the colour over each particle and its pair partners,
    clipped to [0.2, 1] (csf_consistent.py:231-259)."""
    hi, lo = color.copy(), color.copy()
    i, j = pairs[:, 0], pairs[:, 1]
    np.maximum.at(hi, i, color[j])
    np.minimum.at(lo, i, color[j])
    np.maximum.at(hi, j, color[i])
    np.minimum.at(lo, j, color[i])
    return np.clip(hi - lo, color.dtype.type(0.2), color.dtype.type(1.0))


def csf_fields(pos, mass, pairs, h, rho0, normal_smoothing=2, stencil=4.0, curvature_scheme="fit_quadratic",
               curvature_color_smoothing=0, delta_normalization="legacy", wall=None, contact_angle=None,
               contact_angle_reach=2.0):
    """The fields of csf_consistent.py:262-381; with ``wall`` and
    ``contact_angle`` the contact-angle boundary acts on both colour gradients
    (:309-311, :330-332)."""
    T = pos.dtype.type
    vol = (mass / T(rho0)).astype(pos.dtype)
    c = colour(pos, vol, pairs, h)
    m, _ = mls_matrix(pos, vol, pairs, h)
    bc = None
    if wall is not None and contact_angle is not None:
        from .contact_angle import apply_contact_angle_boundary

        def bc(g):
            return apply_contact_angle_boundary(g, pos, wall, h, contact_angle, contact_angle_reach)
    grad_c, mag, normal = _normal(pos, c, vol, pairs, h, m, normal_smoothing, bc)
    if curvature_color_smoothing > 0:
        c_s = np.clip(shepard_smooth(c[:, None], pos, vol, pairs, h, curvature_color_smoothing)[:, 0], T(0), T(1))
        _, _, normal_s = _normal(pos, c_s, vol, pairs, h, m, normal_smoothing, bc)
        kappa = mls_divergence(pos, normal_s, vol, pairs, h, m)
    else:
        kappa = mls_divergence(pos, normal, vol, pairs, h, m)
    delta_s = T(2) * mag if delta_normalization == "legacy" else mag / colour_range(c, pairs)
    if curvature_scheme == "fit_quadratic":
        kappa = fit_curvature_quadratic(pos, normal, delta_s, pairs, h, kappa, stencil=stencil)
    elif curvature_scheme == "fit_circle":
        kappa = fit_curvature_circle(pos, normal, delta_s, pairs, h, kappa, stencil=stencil)
    elif curvature_scheme != "mls":
        raise ValueError(f"unknown curvature_scheme {curvature_scheme!r}")
    return {"color": c, "grad_c": grad_c, "normal": normal, "kappa": kappa, "delta_s": delta_s}


def surface_tension_acceleration(pos, density, mass, h, sigma, rho0, stencil=4.0, pairs=None,
                                 curvature_scheme="fit_quadratic", delta_normalization="legacy", wall=None,
                                 contact_angle=None, contact_angle_reach=2.0, contact_angle_model="rotate"):
    """CSF acceleration of a 2-D fluid cloud and its fields (with a fit, the
    4h pair list is built here, as the reference does); with a wall and a
    contact angle either the normal boundary ("rotate") or the wall-adhesion
    traction ("young", "brackbill") of csf_consistent.py:411-443."""
    T = pos.dtype.type
    if curvature_scheme != "mls" or pairs is None:
        pairs = cell_linked_pairs(pos, stencil * h)
    model = contact_angle_model if contact_angle is not None else None
    rotate = model in (None, "rotate")
    st = csf_fields(pos, mass, pairs, h, rho0, stencil=stencil, curvature_scheme=curvature_scheme,
                    delta_normalization=delta_normalization, wall=wall,
                    contact_angle=contact_angle if rotate else None, contact_angle_reach=contact_angle_reach)
    mag = np.sqrt((st["grad_c"] ** 2).sum(1))
    ds = st["delta_s"].copy()
    ds[mag <= T(1e-3) * mag.max()] = T(0)
    st["delta_s"] = ds
    force = (T(-sigma) * st["kappa"] * ds)[:, None] * st["normal"]
    if model in ("young", "brackbill") and wall is not None:
        from .contact_angle import wall_adhesion_force
        force = force + wall_adhesion_force(pos, wall, st["normal"], contact_angle, sigma, ds, h, model=model)
    return (force / density[:, None]).astype(pos.dtype), st
