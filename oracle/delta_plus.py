"""Oracle (test infrastructure only): the delta-plus step, 2-D and 3-D.

numpy restatement of delta_plus.py:105-229 (``delta_plus_step``) with its
helpers: the fluid geometry of :36-50 (first moment M, eigenvalues, eigen-
floored inverse and the renormalised gradient), the boundary band of :53-69,
the regularisation of :72-76 and the wall tangent of :79-102, plus the
psi-form diffusion of density_diffusion.py:145-172.  h = 2 dx, Wendland C2.
Pairs: unique i < j within 2h (strict), fluid first, wall-wall pairs dropped.

The reference step is 2-D only (delta_plus.py:119).  The same statements are
written here for D = 2 or 3 (read from the positions' shape); for D = 2 every
operation is the reference's.  What D = 3 changes, each a generalisation of a
2-D statement with no 3-D reference to pin it:

* the 3-D Wendland C2 constant 21 / (16 pi h^3) (threed/kernel3.py:139-164);
* Monaghan's radial viscous stress coefficient 2 (D + 2) nu (8 nu in 2-D,
  as the comment at delta_plus.py:185 derives it);
* wall stations of volume dx^D (dx^2 per unit span in 2-D); gravity along -y;
* the D x D first moment and its eigen-decomposition;
* the empty-cap test's tangential distance |ray x n| (the 2-D cross product
  is its z component);
* the wall tangent: a particle whose wall-tangent shift conflicts with the
  interface normal keeps the part of that shift along the line both tangent
  planes share (n_wall x n_surface); in 2-D the two tangent lines share only
  the origin, which is the reference's zero.  Stations at the same distance
  with conflicting normals pin the particle, as in 2-D.
"""
from __future__ import annotations

import math

import numpy as np

from .neighbors import cell_linked_pairs


def wendland_sigma(h, dim=2):
    """Wendland C2 normalisation: 7 / (4 pi h^2) in 2-D (droplet_impact.py:320-346),
    21 / (16 pi h^3) in 3-D (threed/kernel3.py:139-164)."""
    return 7.0 / (4.0 * math.pi * h * h) if dim == 2 else 21.0 / (16.0 * math.pi * h * h * h)


def wendland(r, h, dim=2):
    T = r.dtype.type
    q = r / T(h)
    t = np.maximum(T(1) - T(0.5) * q, T(0))
    return T(wendland_sigma(h, dim)) * t ** 4 * (T(2) * q + T(1))


def wendland_grad(delta, h, eps=1.0e-12):
    T = delta.dtype.type
    dim = delta.shape[1]
    r = np.sqrt((delta * delta).sum(1))
    q = r / T(h)
    t = np.maximum(T(1) - T(0.5) * q, T(0))
    ds = T(-5.0) * q * t ** 3
    scale = T(wendland_sigma(h, dim)) * ds / (T(h) * np.maximum(r, T(eps)))
    return delta * scale[:, None]


def _both(shape, dtype, i, j, at_i, at_j):
    out = np.zeros(shape, dtype=dtype)
    np.add.at(out, i, at_i)
    np.add.at(out, j, at_j)
    return out


def _eigh2(m):
    """Ascending eigenvalues and column eigenvectors of symmetric 2x2 blocks
    (numpy.linalg.eigh, the LAPACK routine torch also calls)."""
    return np.linalg.eigh(m)


def delta_plus_step(pos, velocity, density, mass, *, dx, sound_speed, reference_speed, dt,
                    rho0=1000.0, gravity=9.81, viscosity=1.0e-6, diffusion=0.1, alpha=0.02,
                    wall=None, wall_velocity=None, wall_normal=None, pairs=None):
    T = pos.dtype.type
    dt_ = pos.dtype
    n, D = pos.shape
    h = 2 * dx
    nu_r = 2 * (D + 2) * viscosity + alpha * h * sound_speed
    vol_w = dx ** D   # wall station volume
    if wall is None:
        wall = np.zeros((0, D), dtype=dt_)
    if wall_velocity is None:
        wall_velocity = np.zeros_like(wall)
    if wall_normal is None:
        wall_normal = wall
    wall_normal = wall_normal / np.sqrt((wall_normal ** 2).sum(1))[:, None] if len(wall) else wall_normal
    cloud = np.concatenate((pos, wall))
    if pairs is None:
        pairs = cell_linked_pairs(cloud, 2 * h)
    i, j = pairs[:, 0], pairs[:, 1]
    keep = (i < n) & (((cloud[i] - cloud[j]) ** 2).sum(1) < T((2 * h) ** 2))
    i, j = i[keep], j[keep]
    sep = cloud[i] - cloud[j]
    radius = np.sqrt((sep * sep).sum(1))
    weight = wendland(radius, h, D)
    grad = wendland_grad(sep, h)
    ff = j < n
    a, b, d, g = i[ff], j[ff], sep[ff], grad[ff]
    f, w, dw, gw, ww = i[~ff], j[~ff] - n, sep[~ff], grad[~ff], weight[~ff]
    volume = mass / density
    p = T(sound_speed ** 2) * (density - T(rho0))
    nw = wall.shape[0]
    p_sum = np.zeros(nw, dtype=dt_)
    np.add.at(p_sum, w, ww * (p[f] + density[f] * T(gravity) * dw[:, 1]))
    w_sum = np.zeros(nw, dtype=dt_)
    np.add.at(w_sum, w, ww)
    wall_p = p_sum / np.maximum(w_sum, np.finfo(dt_).tiny)
    wall_rho = T(rho0) + wall_p / T(sound_speed ** 2)
    if (wall_rho[w] <= 0).any():
        raise FloatingPointError("nonpositive extrapolated wall density")
    force = -(volume[a] * volume[b] * (p[a] + p[b]))[:, None] * g
    if nu_r:
        approach = ((velocity[a] - velocity[b]) * d).sum(1)
        pi_ij = approach / np.maximum((d * d).sum(1), T(1.0e-12 * h * h))
        force = force + (T(rho0 * nu_r) * volume[a] * volume[b] * pi_ij)[:, None] * g
    n_wall = wall_normal[w]
    toward = n_wall * np.sign((gw * n_wall).sum(1))[:, None]
    closing = ((velocity[f] - wall_velocity[w]) * toward).sum(1)
    normal_grad = (gw * toward).sum(1)[:, None] * toward
    twice = p[f] + wall_p[w] + T(2) * density[f] * T(sound_speed) * closing
    wall_force = -(volume[f] * T(vol_w) * twice)[:, None] * normal_grad
    net = _both((n, D), dt_, a, b, force, -force)
    np.add.at(net, f, wall_force)
    reaction = np.zeros((nw, D), dtype=dt_)
    np.add.at(reaction, w, -wall_force)
    gvec = np.zeros(D, dtype=dt_)
    gvec[1] = -gravity
    acc = net / mass[:, None] + gvec
    new_v = velocity + T(dt) * acc

    # fluid geometry (delta_plus.py:36-50)
    outer = -d[:, :, None] * g[:, None, :]
    moment = _both((n, D, D), dt_, a, b, volume[b, None, None] * outer, volume[a, None, None] * outer)
    eig, axes = _eigh2(moment)
    floor = np.maximum(T(0.1) * eig.mean(1, keepdims=True), T(1.0e-12))
    inverse = (axes / np.maximum(eig, floor)[:, None, :]) @ np.transpose(axes, (0, 2, 1))

    def gradient(values):
        pg = (values[b] - values[a])[:, None] * g
        s = _both((n, D), dt_, a, b, volume[b, None] * pg, volume[a, None] * pg)
        return (inverse @ s[:, :, None])[:, :, 0]

    lam = eig[:, 0]
    div_pair = ((new_v[b] - new_v[a]) * g).sum(1)
    div = _both((n,), dt_, a, b, volume[b] * div_pair, volume[a] * div_pair)
    normal_speed = ((wall_velocity[w] - new_v[f]) * n_wall).sum(1)
    np.add.at(div, f, T(2 * vol_w) * normal_speed * (n_wall * gw).sum(1))
    rate = -density * div
    if diffusion:
        grad_rho = gradient(density)
        radial = -(d * g).sum(1)
        dist2 = (d * d).sum(1)
        proj = T(0.5) * ((grad_rho[a] + grad_rho[b]) * d).sum(1)
        contrast = (density[a] - density[b]) - proj
        coupling = contrast * radial / (dist2 + T(1.0e-12))
        scale = T(2 * diffusion * h * sound_speed)
        np.add.at(rate, a, -scale * volume[b] * coupling)
        np.add.at(rate, b, scale * volume[a] * coupling)
    new_rho = density + T(dt) * rate
    if not (np.isfinite(new_rho) & (new_rho > 0)).all():
        raise FloatingPointError("delta-plus density became nonpositive or nonfinite")

    # boundary band (delta_plus.py:53-69)
    grad_lam = gradient(lam)
    mag = np.sqrt((grad_lam ** 2).sum(1))
    normal = -grad_lam / np.maximum(mag, T(1.0e-12))[:, None]

    def occupied(ray, direction):
        axial = (ray * direction).sum(1)
        if D == 2:
            tang = np.abs(ray[:, 0] * direction[:, 1] - ray[:, 1] * direction[:, 0])
        else:
            tang = np.sqrt((np.cross(ray, direction) ** 2).sum(1))
        off = ray - T(h) * direction
        return np.where((ray * ray).sum(1) >= T(2 * h * h), (off * off).sum(1) < T(h * h),
                        np.abs(axial - T(h)) + tang < T(h))

    covered = _both((n,), dt_, a, b, occupied(-d, normal[a]).astype(dt_), occupied(d, normal[b]).astype(dt_))
    surface = (lam < 0.2) | ((lam < 0.75) & (covered == 0))
    nb = _both((n,), dt_, a, b, surface[b].astype(dt_), surface[a].astype(dt_))
    band = surface | (nb > 0)
    strength = mag * T(h)

    # positional shift (delta_plus.py:205-226)
    w_ref = wendland(np.array([dx], dtype=dt_), h, D)[0]
    repulsion = (T(1) + T(0.2) * (weight / w_ref) ** 4)[:, None] * grad
    q = repulsion[ff] / (density[a] + density[b])[:, None]
    raw = _both((n, D), dt_, a, b, mass[b, None] * q, -mass[a, None] * q)
    wall_ratio = wall_rho[w] * T(vol_w) / (density[f] + wall_rho[w])
    np.add.at(raw, f, wall_ratio[:, None] * repulsion[~ff])
    raw = raw * T(-(dt * sound_speed / h) * (reference_speed / sound_speed) * (2 * h) ** 2)
    tangent = raw - (raw * normal).sum(1)[:, None] * normal
    resolved = (lam >= 0.55) & (strength > 1.0e-6)
    shift = np.where(band[:, None], np.where(resolved[:, None], tangent, T(0)), raw)

    # wall tangent (delta_plus.py:79-102)
    if f.size:
        dist2 = (dw * dw).sum(1)
        nearest = np.full(n, np.inf, dtype=dt_)
        np.minimum.at(nearest, f, dist2)
        tied = dist2 == nearest[f]
        part, normals = f[tied], n_wall[tied]
        first = np.full(n, part.size, dtype=np.int64)
        np.minimum.at(first, part, np.arange(part.size))
        direction = normals[np.minimum(first, part.size - 1)]
        tan = shift - (shift * direction).sum(1)[:, None] * direction
        tol = T(1.0e-6) * np.sqrt((shift * shift).sum(1))
        conflict = band & (np.abs((tan * normal).sum(1)) > tol)
        other = np.abs((tan[part] * normals).sum(1)) > tol[part]
        pinned = np.zeros(n, dtype=bool)
        np.maximum.at(pinned, part, other)
        if D == 2:
            keep = tan * T(0)
        else:
            # the line both tangent planes share: n_wall x n_surface
            line = np.cross(direction, normal)
            ln = np.sqrt((line * line).sum(1))
            line = np.where((ln > T(1.0e-12))[:, None], line / np.maximum(ln, T(1.0e-30))[:, None], T(0))
            keep = (tan * line).sum(1)[:, None] * line
        constrained = np.where(conflict[:, None], keep, tan)
        constrained = np.where(pinned[:, None], T(0), constrained)
        shift = np.where(np.isfinite(nearest)[:, None], constrained, shift)
    return {"position": pos + T(dt) * new_v + shift, "velocity": new_v, "density": new_rho,
            "acceleration": acc, "wall_reaction": reaction, "shift": shift}
