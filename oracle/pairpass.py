"""Oracle: the WCSPH pair pass in numpy (2-D ``rhs``, ``rhs_3d``, threed ops).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Every function keeps the reference's pair-list scatter structure (``np.add.at``
plays the role of ``index_add``) and computes in the dtype of the positions,
as the reference does.  Citations are to the reference tree:

* kernels ``pair_kernels`` / ``cubic_spline_*``   src/tensorsph/droplet_impact.py:276-371
* Wendland C2                                   src/tensorsph/droplet_impact.py:320-346
* ``tait_pressure``                             src/tensorsph/droplet_impact.py:415-427
* ``rhs`` (2-D)                                  src/tensorsph/droplet_impact.py:810-1228
* ``rhs_3d``                                     src/tensorsph/dam_break_3d.py:290-422
* diffusion (Molteni, Antuono psi)              src/tensorsph/density_diffusion.py:78-197
* threed ``accelerations`` and parts            src/tensorsph/threed/operators3.py:51-295
* 3-D kernel + Laplacian                        src/tensorsph/threed/kernel3.py:48-181
* ``shift_positions``                           src/tensorsph/particle_shifting.py:93-224
"""
from __future__ import annotations

import math

import numpy as np

from .neighbors import cell_linked_pairs, minimum_image

VISCOUS_LAPLACIAN_FACTOR = 2.0


def _t(x, like):
    return np.asarray(x, dtype=like.dtype)


def norm(delta):
    acc = delta[..., 0] * delta[..., 0]
    for a in range(1, delta.shape[-1]):
        acc = acc + delta[..., a] * delta[..., a]
    return np.sqrt(acc)


# ----------------------------------------------------------------- kernels ---

def sigma_cubic(h, dim):
    return 10.0 / (7.0 * math.pi * h * h) if dim == 2 else 1.0 / (math.pi * h ** 3)


def shape(q):
    first = 1.0 - 1.5 * q * q + 0.75 * q ** 3
    second = 0.25 * np.maximum(2.0 - q, 0) ** 3
    return np.where(q < 1.0, first, np.where(q < 2.0, second, 0.0)).astype(q.dtype)


def shape_prime(q):
    return np.where(q < 1.0, -3.0 * q + 2.25 * q * q,
                    np.where(q < 2.0, -0.75 * (2.0 - q) ** 2, 0.0)).astype(q.dtype)


def shape_second(q):
    return np.where(q < 1.0, -3.0 + 4.5 * q,
                    np.where(q < 2.0, 1.5 * (2.0 - q), 0.0)).astype(q.dtype)


def cubic_kernel(r, h, dim):
    dt = r.dtype.type
    q = r / dt(h)
    return dt(sigma_cubic(h, dim)) * np.maximum(shape(q), dt(0))


def cubic_pair_kernels(delta, h, dim, eps=1.0e-12):
    """``(W, grad_i W)`` for ``delta = x_i - x_j`` (droplet_impact.py:349-371)."""
    dt = delta.dtype.type
    r = norm(delta)
    q = r / dt(h)
    sig = dt(sigma_cubic(h, dim))
    weight = sig * np.maximum(shape(q), dt(0))
    scale = sig * shape_prime(q) / (dt(h) * np.maximum(r, dt(eps)))
    return weight, delta * scale[..., None]


def cubic_laplacian_3d(delta, h, eps=1.0e-12):
    """``laplacian_i W`` in 3-D with the closed r -> 0 limit (kernel3.py:108-124)."""
    dt = delta.dtype.type
    r = norm(delta)
    q = r / dt(h)
    twice = np.where(q > 1.0e-10, 2.0 * shape_prime(q) / np.maximum(q, dt(eps)),
                     dt(-6.0)).astype(delta.dtype)
    radial = shape_second(q) + twice
    sig = dt(sigma_cubic(h, 3))
    return np.where(q < 2.0, sig * radial / dt(h * h), dt(0)).astype(delta.dtype)


def wendland(r, h, dim):
    dt = r.dtype.type
    q = r / dt(h)
    sig = 7.0 / (4.0 * math.pi * h * h) if dim == 2 else 21.0 / (16.0 * math.pi * h ** 3)
    t = np.maximum(1.0 - 0.5 * q, 0.0).astype(r.dtype)
    return dt(sig) * t ** 4 * (2.0 * q + 1.0)


def wendland_gradient(delta, h, dim, eps=1.0e-12):
    dt = delta.dtype.type
    r = norm(delta)
    q = r / dt(h)
    sig = 7.0 / (4.0 * math.pi * h * h) if dim == 2 else 21.0 / (16.0 * math.pi * h ** 3)
    t = np.maximum(1.0 - 0.5 * q, 0.0).astype(delta.dtype)
    scale = dt(sig) * (-5.0 * q * t ** 3) / (dt(h) * np.maximum(r, dt(eps)))
    return delta * scale[..., None]


# --------------------------------------------------------------------- EOS ---

def tait(rho, rho0, c0, gamma, ratio_floor=0.01):
    """Clamped Tait law; ``ratio_floor=None`` is the threed variant."""
    dt = rho.dtype.type
    bulk = rho0 * c0 ** 2 / gamma
    ratio = rho / dt(rho0)
    if ratio_floor is not None:
        ratio = np.maximum(ratio, dt(ratio_floor))
    return np.maximum(dt(bulk) * (ratio ** dt(gamma) - dt(1.0)), dt(0))


def tait_inverse(p, rho0, c0, gamma, clamp_rho0=True):
    dt = p.dtype.type
    bulk = rho0 * c0 ** 2 / gamma
    if clamp_rho0:
        out = dt(rho0) * (p / dt(bulk) + dt(1.0)) ** dt(1.0 / gamma)
        return np.maximum(out, dt(rho0))
    return dt(rho0) * (dt(1.0) + np.maximum(p, dt(0)) / dt(bulk)) ** dt(1.0 / gamma)


# -------------------------------------------------------------- diffusion ---

def _sym_eig_floor_solve(moment, rhs_vec, floor_frac, mean_clamp=1.0e-30):
    """``(V diag(max(l, f)) V^T)^-1 g`` with ``f = floor * trace/D`` per row."""
    vals, vecs = np.linalg.eigh(moment)
    dim = moment.shape[-1]
    trace = vals.sum(axis=-1)
    mean = np.maximum(trace / dim, mean_clamp)
    floor = (floor_frac * mean)[..., None]
    clamped = np.maximum(vals, floor)
    proj = np.einsum("pka,pk->pa", vecs, rhs_vec)
    out = np.einsum("pak,pk->pa", vecs, proj / clamped)
    out[trace <= 0.0] = 0.0
    return out.astype(moment.dtype)


def molteni_rate(rho, mass, radial, dist2, i, j, scale):
    dt = rho.dtype.type
    vi, vj = mass[i] / rho[i], mass[j] / rho[j]
    coupling = (rho[i] - rho[j]) * radial / (dist2 + dt(1.0e-12))
    rate = np.zeros_like(rho)
    np.add.at(rate, i, -dt(scale) * vj * coupling)
    np.add.at(rate, j, dt(scale) * vi * coupling)
    return rate


def renormalized_gradient(n, dim, rho, mass, i, j, delta, grad_w, floor):
    dt = rho.dtype
    vi, vj = mass[i] / rho[i], mass[j] / rho[j]
    diff = (rho[j] - rho[i])[:, None]
    g = np.zeros((n, dim), dtype=dt)
    np.add.at(g, i, vj[:, None] * diff * grad_w)
    np.add.at(g, j, vi[:, None] * diff * grad_w)
    outer = -(delta[:, :, None] * grad_w[:, None, :])
    m = np.zeros((n, dim, dim), dtype=dt)
    np.add.at(m, i, vj[:, None, None] * outer)
    np.add.at(m, j, vi[:, None, None] * outer)
    return _sym_eig_floor_solve(m.astype(np.float64), g.astype(np.float64), floor).astype(dt)


def antuono_rate(rho, mass, delta, radial, dist2, i, j, scale, grad_rho):
    dt = rho.dtype.type
    vi, vj = mass[i] / rho[i], mass[j] / rho[j]
    projected = dt(0.5) * ((grad_rho[i] + grad_rho[j]) * delta).sum(axis=1)
    contrast = (rho[i] - rho[j]) - projected
    coupling = contrast * radial / (dist2 + dt(1.0e-12))
    rate = np.zeros_like(rho)
    np.add.at(rate, i, -dt(scale) * vj * coupling)
    np.add.at(rate, j, dt(scale) * vi * coupling)
    return rate


# ------------------------------------------------------------------ 2-D rhs ---

def compression_sums(all_mass, rho0, w_self, i, j, wij, n, inverse_reference):
    """S_a = W(0) Vref_a + Kref sum_b W_ab Vref_b over the fluid rows, Vref =
    m / rho0, Kref on the neighbour term only (compression_regularization.py:
    96-139)."""
    vol = all_mass / all_mass.dtype.type(rho0)
    sums = all_mass.dtype.type(w_self) * vol[:n]
    weighted = all_mass.dtype.type(inverse_reference) * wij
    np.add.at(sums, i, weighted * vol[j])
    back = j < n
    np.add.at(sums, j[back], weighted[back] * vol[i[back]])
    return sums


def average_inverse_reference(sums):
    """(1 / mean{S : S > 1}, count), 1 for an empty set
    (compression_regularization.py:142-161)."""
    mask = sums > 1.0
    counted = int(mask.sum())
    if counted == 0:
        return 1.0, 0
    total = float(sums[mask].sum())
    if total <= 0.0:
        return 1.0, 0
    return counted / total, counted


def free_surface_pressure(rho, pressure, delta, wij, i, j, cfg):
    """Adami's extrapolation onto particles with rho < threshold rho0 over the
    fluid pairs (droplet_impact.py:429-492): "interior" donors in
    surface_pressure_layers Jacobi passes, "all" in one."""
    T = pressure.dtype.type
    n = pressure.shape[0]
    known = ~(rho < T(cfg.surface_pressure_threshold * cfg.rho0))
    p = pressure.copy()
    grav = T(cfg.gravity) * delta[:, 1]
    literal = cfg.surface_pressure_donors == "all"
    for _ in range(1 if literal else max(1, cfg.surface_pressure_layers)):
        receive = ~known
        if not receive.any():
            break
        w_i = wij if literal else wij * known[j].astype(wij.dtype)
        w_j = wij if literal else wij * known[i].astype(wij.dtype)
        num = np.zeros(n, dtype=p.dtype)
        den = np.zeros(n, dtype=p.dtype)
        np.add.at(num, i, w_i * (p[j] - grav * rho[j]))
        np.add.at(den, i, w_i)
        np.add.at(num, j, w_j * (p[i] + grav * rho[i]))
        np.add.at(den, j, w_j)
        filled = receive & (den > T(1.0e-30))
        p = np.where(filled, np.maximum(num / np.maximum(den, T(1.0e-30)), T(0)), p)
        known = known | filled
    return p


def rhs(pos, vel, mass, cfg, pairs=None, wall=None, dt=None, wall_vel=None,
        wall_accel=None, split=False, wrap_width=None, nu_field=None,
        density_offset=None, state=None):
    """2-D WCSPH right-hand side (droplet_impact.py:810-1228).

    ``cfg`` is any object with the reference ``Config`` attributes.  With
    ``density_regularization="compression"`` the inverse reference
    compression is read from and written to ``state["inverse_reference"]``
    (1 when absent), the count to ``state["counted"]``.
    """
    T = pos.dtype.type
    h = cfg.h_factor * cfg.dx
    n, dim = pos.shape
    step_dt = cfg.dt if dt is None else float(dt)
    if dim != 2:
        raise ValueError("rhs implements 2-D smoothing only")
    unit = lattice_mass_unit_2d(cfg)
    if wall is None:
        all_pos, all_mass, nw = pos, mass, 0
    else:
        nw = wall.shape[0]
        all_pos = np.concatenate((pos, wall))
        all_mass = np.concatenate((mass, np.full(nw, unit, dtype=pos.dtype)))
    if pairs is None:
        pairs = cell_linked_pairs(all_pos, 2.0 * h)
        keep = (pairs[:, 0] < n) | (pairs[:, 1] < n)
        pairs = pairs[keep]
    w0 = T(sigma_cubic(h, 2))
    rho_all = np.zeros(n + nw, dtype=pos.dtype)
    rho_all[:n] = mass * cubic_kernel(np.zeros(n, dtype=pos.dtype), h, 2)
    gravity = np.zeros_like(pos)
    gravity[:, 1] = -T(cfg.gravity)
    if pairs.shape[0] == 0:
        rho = np.maximum(rho_all[:n], T(0.1 * cfg.rho0))
        return rho, tait(rho, cfg.rho0, cfg.sound_speed, cfg.gamma), gravity
    i, j = pairs[:, 0], pairs[:, 1]
    delta = all_pos[i] - all_pos[j]
    if wrap_width is not None:
        width = T(wrap_width)
        delta = np.stack((delta[:, 0] - width * np.round(delta[:, 0] / width), delta[:, 1]), 1)
    distance = norm(delta)
    wij, grad_w = cubic_pair_kernels(delta, h, 2)
    np.add.at(rho_all, i, all_mass[j] * wij)
    np.add.at(rho_all, j, all_mass[i] * wij)
    rho = np.maximum(rho_all[:n], T(0.1 * cfg.rho0))
    if density_offset is not None:
        rho = np.maximum(rho + density_offset, T(0.1 * cfg.rho0))
    if cfg.density_renormalization:
        total = np.zeros(n + nw, dtype=pos.dtype)
        np.add.at(total, i, wij)
        np.add.at(total, j, wij)
        total[:n] = total[:n] + w0
        s_full = lattice_kernel_sum_2d(h, cfg.dx)
        rho = np.maximum(rho * (T(s_full) / np.maximum(total[:n], T(1.0e-12))), T(0.1 * cfg.rho0))
    if cfg.density_diffusion > 0.0:
        ff = (i < n) & (j < n)
        radial = -(delta[ff] * grad_w[ff]).sum(axis=1)
        scale = 2.0 * cfg.density_diffusion * cfg.sound_speed * cfg.h_factor * cfg.dx
        if cfg.density_diffusion_form == "molteni":
            rate = molteni_rate(rho, mass, radial, distance[ff] ** 2, i[ff], j[ff], scale)
        else:
            grad_rho = renormalized_gradient(n, 2, rho, mass, i[ff], j[ff], delta[ff],
                                             grad_w[ff], cfg.density_diffusion_eigenvalue_floor)
            rate = antuono_rate(rho, mass, delta[ff], radial, distance[ff] ** 2,
                                i[ff], j[ff], scale, grad_rho)
        rho = np.maximum(rho + T(step_dt) * rate, T(0.1 * cfg.rho0))
    if getattr(cfg, "density_regularization", "none") == "compression":
        state = {} if state is None else state
        used = (state.get("inverse_reference", 1.0)
                if cfg.compression_normalization == "reference_mean" else 1.0)
        sums = compression_sums(all_mass, cfg.rho0, w0, i, j, wij, n, used)
        state["inverse_reference"], state["counted"] = average_inverse_reference(sums)
        if cfg.compression_regularization_rule == "free_surface":
            sums = np.maximum(sums, T(1))
        rho = np.maximum(sums * T(cfg.rho0), T(0.1 * cfg.rho0))
    pressure = tait(rho, cfg.rho0, cfg.sound_speed, cfg.gamma)
    if getattr(cfg, "surface_pressure_closure", False):
        ff = (i < n) & (j < n)
        pressure = free_surface_pressure(rho, pressure, delta[ff], wij[ff], i[ff], j[ff], cfg)
    wall_pressure = np.zeros(nw, dtype=pos.dtype)
    if nw:
        i_fluid = i < n
        crossing = i_fluid != (j < n)
        fluid_idx = np.where(i_fluid, i, j)
        wall_idx = np.clip(np.where(i_fluid, j, i) - n, 0, nw - 1)
        weight = np.where(crossing, wij, T(0))
        dy = np.where(i_fluid, -delta[:, 1], delta[:, 1])
        body = -T(cfg.gravity) * dy
        if wall_accel is not None:
            dxw = np.where(i_fluid, -delta[:, 0], delta[:, 0])
            body = body - (wall_accel[wall_idx, 0] * dxw + wall_accel[wall_idx, 1] * dy)

        def extrapolate(p_vec, r_vec):
            zeros = np.zeros(nw, dtype=pos.dtype)
            source = np.concatenate((p_vec, zeros))[fluid_idx]
            if cfg.gravity != 0.0:
                source = source + np.concatenate((r_vec, zeros))[fluid_idx] * body
            num = np.zeros(nw, dtype=pos.dtype)
            den = np.zeros(nw, dtype=pos.dtype)
            np.add.at(num, wall_idx, source * weight)
            np.add.at(den, wall_idx, weight)
            p_w = np.maximum(num / np.maximum(den, T(1.0e-30)), T(0))
            return p_w, tait_inverse(p_w, cfg.rho0, cfg.sound_speed, cfg.gamma)

        wall_pressure, wall_density = extrapolate(pressure, rho)
        if cfg.boundary_consistent_density:
            mw = all_mass[n:]
            dmass = mw * (wall_density / T(cfg.rho0)) - mw
            corr = np.zeros(n, dtype=pos.dtype)
            np.add.at(corr, fluid_idx[crossing], dmass[wall_idx[crossing]] * wij[crossing])
            rho = np.maximum(rho + corr, T(0.1 * cfg.rho0))
            pressure = tait(rho, cfg.rho0, cfg.sound_speed, cfg.gamma)
            wall_pressure, wall_density = extrapolate(pressure, rho)
        p_all = np.concatenate((pressure, wall_pressure))
        d_all = np.concatenate((rho, wall_density))
        wv = np.zeros((nw, 2), dtype=pos.dtype) if wall_vel is None else wall_vel
        all_vel = np.concatenate((vel, wv))
    else:
        p_all, d_all, all_vel = pressure, rho, vel
    term = p_all[i] / (d_all[i] * d_all[i]) + p_all[j] / (d_all[j] * d_all[j])
    pair_p = term[:, None] * grad_w
    acc = np.zeros((n + nw, 2), dtype=pos.dtype)
    np.add.at(acc, i, -all_mass[j, None] * pair_p)
    np.add.at(acc, j, all_mass[i, None] * pair_p)
    fluid_pair = (i < n) & (j < n)
    if nu_field is None:
        nu = T(cfg.viscosity)
    else:
        pad = np.concatenate((nu_field, np.zeros(nw, dtype=pos.dtype)))
        nu = np.where(fluid_pair, T(0.5) * (pad[i] + pad[j]), np.where(i < n, pad[i], pad[j]))
    if nw and cfg.wall_friction > 0.0:
        cross = (i < n) ^ (j < n)
        blend = fluid_pair.astype(pos.dtype) + T(cfg.wall_friction) * cross.astype(pos.dtype)
        vscale = (T(2.0) * nu * blend)[:, None]
    elif nw:
        vscale = (T(2.0) * nu * fluid_pair.astype(pos.dtype))[:, None]
    else:
        vscale = T(2.0) * nu
        if nu_field is not None:
            vscale = vscale[:, None]
    dv = all_vel[i] - all_vel[j]
    lw = np.maximum(-(delta * grad_w).sum(axis=1), T(0)) / (distance * distance + T(0.01 * h * h))
    visc_i = -vscale * dv * (all_mass[j] / d_all[j] * lw)[:, None]
    visc_j = vscale * dv * (all_mass[i] / d_all[i] * lw)[:, None]
    av = np.zeros((n + nw, 2), dtype=pos.dtype)
    np.add.at(av, i, visc_i)
    np.add.at(av, j, visc_j)
    total = acc[:n] + av[:n] + gravity
    if not split:
        return rho, pressure, total
    reaction = np.zeros((nw, 2), dtype=pos.dtype)
    if nw:
        i_fluid = i < n
        crossing = i_fluid != (j < n)
        wall_idx = np.clip(np.where(i_fluid, j, i) - n, 0, nw - 1)
        sign = np.where(i_fluid, T(-1), T(1))
        pm = all_mass[i] * all_mass[j]
        np.add.at(reaction, wall_idx, -sign[:, None] * pm[:, None] * pair_p
                  * crossing[:, None].astype(pos.dtype))
        if cfg.wall_friction > 0.0:
            vf = np.where(i_fluid[:, None], visc_i, visc_j)
            fm = np.where(i_fluid, all_mass[i], all_mass[j])
            np.add.at(reaction, wall_idx, -vf * fm[:, None] * crossing[:, None].astype(pos.dtype))
    return rho, pressure, total, {"reaction": reaction, "face_pressure": wall_pressure}


def lattice_kernel_sum_2d(h, dx):
    reach = int(math.ceil(2.0 * h / dx)) + 1
    off = np.arange(-reach, reach + 1, dtype=np.float64) * dx
    gx, gy = np.meshgrid(off, off, indexing="xy")
    r = np.sqrt(gx * gx + gy * gy).reshape(-1)
    return float(cubic_kernel(r, h, 2).sum())


def lattice_mass_unit_2d(cfg):
    if cfg.density_calibration:
        return float(cfg.rho0 / lattice_kernel_sum_2d(cfg.h_factor * cfg.dx, cfg.dx))
    return cfg.rho0 * cfg.dx * cfg.dx


def lattice_kernel_sum_3d(dx, h, half_width=None):
    if half_width is None:
        half_width = int(math.ceil(2.0 * h / dx)) + 1
    n = np.arange(-half_width, half_width + 1, dtype=np.float64) * dx
    g = np.stack(np.meshgrid(n, n, n, indexing="ij"), -1).reshape(-1, 3)
    r = np.sqrt((g * g).sum(1))
    return float(cubic_kernel(r, h, 3).sum() * dx ** 3)


def calibrated_mass_3d(dx, h, rho0):
    return rho0 * dx ** 3 / lattice_kernel_sum_3d(dx, h)


def mass_3d(cfg):
    if cfg.density_calibration:
        return calibrated_mass_3d(cfg.dx, cfg.h_factor * cfg.dx, cfg.rho0)
    return cfg.rho0 * cfg.dx ** 3


# ------------------------------------------------------------------ 3-D rhs ---

def rhs_3d(pos, vel, mass, cfg, pairs=None, wall=None, dt=None, return_wall_force=False):
    """3-D WCSPH right-hand side (dam_break_3d.py:290-422)."""
    T = pos.dtype.type
    n = pos.shape[0]
    nw = 0 if wall is None else wall.shape[0]
    h = cfg.h_factor * cfg.dx
    step_dt = cfg.dt if dt is None else dt
    g = np.array([0.0, -cfg.gravity, 0.0], dtype=pos.dtype)
    if wall is not None:
        all_pos = np.concatenate((pos, wall))
        all_mass = np.concatenate((mass, np.full(nw, mass_3d(cfg), dtype=pos.dtype)))
    else:
        all_pos, all_mass = pos, mass
    if pairs is None:
        pairs = cell_linked_pairs(all_pos, 2.0 * h)
    i, j = pairs[:, 0], pairs[:, 1]
    delta = all_pos[i] - all_pos[j]
    distance = norm(delta)
    wij, grad_w = cubic_pair_kernels(delta, h, 3)
    rho_all = all_mass / T(math.pi * h ** 3)
    np.add.at(rho_all, i, all_mass[j] * wij)
    np.add.at(rho_all, j, all_mass[i] * wij)
    rho = np.maximum(rho_all[:n], T(0.1 * cfg.rho0))
    if cfg.density_diffusion > 0.0:
        if cfg.density_diffusion_form != "molteni":
            raise ValueError("rhs_3d implements the 'molteni' form only")
        ff = (i < n) & (j < n)
        radial = -(delta[ff] * grad_w[ff]).sum(axis=1)
        scale = 2.0 * cfg.density_diffusion * cfg.sound_speed * cfg.h_factor * cfg.dx
        rate = molteni_rate(rho, mass, radial, distance[ff] ** 2, i[ff], j[ff], scale)
        rho = np.maximum(rho + T(step_dt) * rate, T(0.1 * cfg.rho0))
    pressure = tait(rho, cfg.rho0, cfg.sound_speed, cfg.gamma)
    if getattr(cfg, "surface_pressure_closure", False):
        # dam_break_3d.py:339-342
        ff = (i < n) & (j < n)
        pressure = free_surface_pressure(rho, pressure, delta[ff], wij[ff], i[ff], j[ff], cfg)
    if nw:
        i_fluid = i < n
        crossing = i_fluid != (j < n)
        fluid_idx = np.where(i_fluid, i, j)
        wall_idx = np.clip(np.where(i_fluid, j, i) - n, 0, nw - 1)
        weight = np.where(crossing, wij, T(0))
        zeros = np.zeros(nw, dtype=pos.dtype)
        dy = np.where(i_fluid, -delta[:, 1], delta[:, 1])
        body = -T(cfg.gravity) * dy
        source = np.concatenate((pressure, zeros))[fluid_idx]
        if cfg.gravity != 0.0:
            source = source + np.concatenate((rho, zeros))[fluid_idx] * body
        num = np.zeros(nw, dtype=pos.dtype)
        den = np.zeros(nw, dtype=pos.dtype)
        np.add.at(num, wall_idx, source * weight)
        np.add.at(den, wall_idx, weight)
        wp = np.maximum(num / np.maximum(den, T(1.0e-30)), T(0))
        wd = tait_inverse(wp, cfg.rho0, cfg.sound_speed, cfg.gamma)
        p_all = np.concatenate((pressure, wp))
        d_all = np.concatenate((rho, wd))
        all_vel = np.concatenate((vel, np.zeros((nw, 3), dtype=pos.dtype)))
    else:
        p_all, d_all, all_vel = pressure, rho, vel
    term = p_all[i] / (d_all[i] * d_all[i]) + p_all[j] / (d_all[j] * d_all[j])
    pair_p = term[:, None] * grad_w
    acc = np.zeros((n + nw, 3), dtype=pos.dtype)
    np.add.at(acc, i, -all_mass[j, None] * pair_p)
    np.add.at(acc, j, all_mass[i, None] * pair_p)
    fluid_pair = (i < n) & (j < n)
    if nw and cfg.wall_friction > 0.0:
        cross = (i < n) ^ (j < n)
        blend = fluid_pair.astype(pos.dtype) + T(cfg.wall_friction) * cross.astype(pos.dtype)
        vscale = (T(2.0 * cfg.viscosity) * blend)[:, None]
    elif nw:
        vscale = (T(2.0 * cfg.viscosity) * fluid_pair.astype(pos.dtype))[:, None]
    else:
        vscale = T(2.0 * cfg.viscosity)
    dv = all_vel[i] - all_vel[j]
    lw = np.maximum(-(delta * grad_w).sum(axis=1), T(0)) / (distance * distance + T(0.01 * h * h))
    visc_i = -vscale * dv * (all_mass[j] / d_all[j] * lw)[:, None]
    visc_j = vscale * dv * (all_mass[i] / d_all[i] * lw)[:, None]
    av = np.zeros((n + nw, 3), dtype=pos.dtype)
    np.add.at(av, i, visc_i)
    np.add.at(av, j, visc_j)
    total = acc[:n] + av[:n] + g
    if not return_wall_force:
        return rho, pressure, total
    reaction = np.zeros((nw, 3), dtype=pos.dtype)
    if nw:
        sign = np.where(i_fluid, T(1), T(-1))
        pf = (sign * all_mass[i] * all_mass[j])[:, None] * pair_p
        fv = np.where(i_fluid[:, None], visc_i, visc_j)
        load = pf - all_mass[fluid_idx, None] * fv
        np.add.at(reaction, wall_idx[crossing], load[crossing])
    return rho, pressure, total, reaction


# ------------------------------------------------------ threed operators ---

def pair_geometry(pos, pairs, h, box=None):
    delta = pos[pairs[:, 0]] - pos[pairs[:, 1]]
    if box is not None:
        delta = minimum_image(delta, box)
    w, g = cubic_pair_kernels(delta, h, 3)
    lap = cubic_laplacian_3d(delta, h)
    return delta, w, g, lap


def accelerations(pos, vel, mass, h, pairs, *, rho0, sound_speed, gamma=7.0,
                  viscosity=0.0, gravity=None, box=None, n_fluid=None,
                  renormalise=True, wall_model="adami", viscous_order=2,
                  density_diffusion=0.0, dt=None, density_diffusion_form="antuono",
                  density_diffusion_eigenvalue_floor=0.1):
    """threed ``accelerations`` (operators3.py:212-256); returns (acc, rho, p)."""
    T = pos.dtype.type
    n, dim = pos.shape
    nf = n if n_fluid is None else n_fluid
    i, j = pairs[:, 0], pairs[:, 1]
    delta, w, gw, lap = pair_geometry(pos, pairs, h, box)
    rho = np.zeros(n, dtype=pos.dtype)
    np.add.at(rho, i, mass[j] * w)
    np.add.at(rho, j, mass[i] * w)
    rho = rho + mass * T(sigma_cubic(h, 3))
    if density_diffusion > 0.0:
        if dt is None or dt <= 0.0:
            raise ValueError("density_diffusion > 0 requires a positive dt")
        ii, jj, dd, gg = i, j, delta, gw
        if n_fluid is not None and n_fluid < n:
            m = (i < n_fluid) & (j < n_fluid)
            ii, jj, dd, gg = i[m], j[m], delta[m], gw[m]
        d2 = (dd * dd).sum(axis=1)
        radial = -(dd * gg).sum(axis=1)
        scale = 2.0 * density_diffusion * sound_speed * h
        if density_diffusion_form == "molteni":
            rate = molteni_rate(rho, mass, radial, d2, ii, jj, scale)
        else:
            grad_rho = renormalized_gradient(n, dim, rho, mass, ii, jj, dd, gg,
                                             density_diffusion_eigenvalue_floor)
            rate = antuono_rate(rho, mass, dd, radial, d2, ii, jj, scale, grad_rho)
        rho = np.maximum(rho + T(dt) * rate, T(0.1 * rho0))
    pressure = tait(rho, rho0, sound_speed, gamma, ratio_floor=None)
    rho_used = rho
    if nf < n and wall_model == "adami":
        ff = (i < nf) & (j >= nf)
        wf = (j < nf) & (i >= nf)
        f = np.concatenate((i[ff], j[wf]))
        wi = np.concatenate((j[ff], i[wf]))
        weight = cubic_kernel(norm(pos[f] - pos[wi]), h, 3)
        if gravity is not None:
            gv = np.asarray(gravity, dtype=pos.dtype).reshape(1, -1)
            donor = pressure[f] + rho[f] * ((pos[wi] - pos[f]) * gv).sum(axis=1)
        else:
            donor = pressure[f]
        num = np.zeros(n, dtype=pos.dtype)
        den = np.zeros(n, dtype=pos.dtype)
        np.add.at(num, wi, donor * weight)
        np.add.at(den, wi, weight)
        out = np.where(den > 0.0, num / np.maximum(den, T(1.0e-30)), T(0))
        p_wall = np.maximum(out[nf:], T(0))
        pressure = np.concatenate((pressure[:nf], p_wall))
        rho_used = np.concatenate((rho[:nf], tait_inverse(p_wall, rho0, sound_speed, gamma,
                                                           clamp_rho0=False)))
    elif nf < n and wall_model != "tait":
        raise ValueError(f"unknown wall_model {wall_model!r}")
    sym = pressure[i] / (rho_used[i] * rho_used[i]) + pressure[j] / (rho_used[j] * rho_used[j])
    acc = np.zeros_like(pos)
    np.add.at(acc, i, -(gw * (mass[j] * sym)[:, None]))
    np.add.at(acc, j, gw * (mass[i] * sym)[:, None])
    if viscosity != 0.0:
        rij = T(0.5) * (rho_used[i] + rho_used[j])
        weight = mass[j] * lap / rij
        r2 = (delta * delta).sum(axis=1)
        vj, vi = mass[j] / rij, mass[i] / rij
        moment = np.zeros(n, dtype=pos.dtype)
        np.add.at(moment, i, r2 * lap * vj)
        np.add.at(moment, j, r2 * lap * vi)
        moment = moment / T(3.0)
        if renormalise:
            weight = weight * (T(2.0) / np.maximum(T(0.5) * (moment[i] + moment[j]), T(1.0e-12)))

        def pair_lap(field, wgt):
            dv = (field[j] - field[i]) * wgt[:, None]
            out = np.zeros_like(field)
            np.add.at(out, i, dv)
            np.add.at(out, j, -dv)
            return out

        va = pair_lap(vel, weight)
        if viscous_order == 4:
            fourth = np.zeros(n, dtype=pos.dtype)
            np.add.at(fourth, i, r2 * r2 * lap * vj)
            np.add.at(fourth, j, r2 * r2 * lap * vi)
            beta = T(0.5) * (fourth[i] + fourth[j]) / T(120.0)
            va = va - pair_lap(va, weight * beta)
        acc = acc + va * T(viscosity)
    if gravity is not None:
        acc[:nf] = acc[:nf] + np.asarray(gravity, dtype=pos.dtype).reshape(1, -1)
    return acc, rho, pressure


# --------------------------------------------------------------- shifting ---

def shift_positions(pos, volume, h, *, dt, v_ref, strength=1.0, limit=0.25,
                    free_surface=0.95, pairs=None, c_reference=None):
    """Lind shifting (particle_shifting.py:166-224); returns (new_pos, state)."""
    T = pos.dtype.type
    n = pos.shape[0]
    if pairs is None:
        pairs = cell_linked_pairs(pos, 2.0 * h)
    c = volume * cubic_kernel(np.zeros(n, dtype=pos.dtype), h, 2)
    grad = np.zeros_like(pos)
    if pairs.shape[0]:
        i, j = pairs[:, 0], pairs[:, 1]
        r = norm(pos[i] - pos[j])
        w = cubic_kernel(r, h, 2)
        np.add.at(c, i, volume[j] * w)
        np.add.at(c, j, volume[i] * w)
        _, gw = cubic_pair_kernels(pos[i] - pos[j], h, 2)
        diff = (c[j] - c[i])[:, None] * gw
        np.add.at(grad, i, volume[j, None] * diff)
        np.add.at(grad, j, volume[i, None] * diff)
    mag = norm(grad)
    normal = np.where(mag[:, None] > 1.0e-30, -grad / np.maximum(mag, T(1.0e-30))[:, None], T(0))
    c_ref = (float(np.quantile(c.astype(np.float64), 0.95)) if c_reference is None
             else float(c_reference))
    fs = c < T(free_surface * c_ref) if c_ref > 0 else np.zeros(n, dtype=bool)
    magnitude = float(strength) * h * float(v_ref) * float(dt)
    shift = -T(magnitude) * grad
    if fs.any():
        nh = normal[fs]
        proj = (shift[fs] * nh).sum(axis=-1, keepdims=True) * nh
        shift[fs] = shift[fs] - proj
    cap = T(float(limit) * h)
    smag = norm(shift)
    clipped = smag > cap
    if clipped.any():
        scale = np.where(clipped, cap / np.maximum(smag, T(1e-300) if T is np.float64 else T(0)),
                         T(1))
        shift = shift * scale[:, None]
    return pos + shift, {"concentration": c, "grad_c": grad, "normal": normal,
                         "shift": shift, "free_surface": fs, "c_reference": c_ref,
                         "magnitude": magnitude}
