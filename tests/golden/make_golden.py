"""Generate golden input/output fixtures by running the reference TensorSPH.

Run in a checkout that has the reference source tree (not on the GPU host):

    python tests/golden/make_golden.py /path/to/TensorSPH/src

Every case seeds its own ``torch.Generator``; inputs and the reference's
outputs are stored together in one ``.npz`` per case family, with the torch
version that produced them.  The committed fixtures are what the oracle and
the CUDA path are pinned against.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import torch

OUT = Path(__file__).resolve().parent


def _np(t):
    return t.detach().cpu().numpy()


def capture_order(fn, *args):
    """Run ``fn`` and record the first stable ``torch.argsort`` it performs.

    ``cell_linked_pairs`` / ``periodic_pairs`` sort the particles by cell with
    one stable argsort before they expand candidates; that permutation is the
    cell order the CUDA counting sort must reproduce bit for bit.
    """
    seen = []
    real = torch.argsort

    def spy(*a, **k):
        out = real(*a, **k)
        if k.get("stable") and not seen:
            seen.append(out.clone())
        return out

    torch.argsort = spy
    try:
        result = fn(*args)
    finally:
        torch.argsort = real
    return result, (seen[0] if seen else torch.empty(0, dtype=torch.long))


def pairs_cases(ns):
    data = {}
    k = 0
    for dim in (1, 2, 3):
        for dtype in (torch.float32, torch.float64):
            for seed in (0, 7):
                g = torch.Generator().manual_seed(seed + 100 * dim)
                pos = (4.0 * torch.randn((301, dim), generator=g)).to(dtype)
                pos[1] = pos[0]
                pos[2] = pos[0] + 0.25 * torch.nn.functional.one_hot(
                    torch.tensor(0), num_classes=dim).to(dtype)
                for cutoff in (0.25, 0.7):
                    pairs, order = capture_order(ns.cell_linked_pairs, pos, cutoff)
                    brute = ns.brute_force_pairs(pos, cutoff)
                    assert torch.equal(pairs, brute)
                    data[f"c{k}_pos"] = _np(pos)
                    data[f"c{k}_cutoff"] = np.float64(cutoff)
                    data[f"c{k}_pairs"] = _np(pairs)
                    data[f"c{k}_order"] = _np(order)
                    k += 1
    # uniform clouds exercise dense cells; lattice points sit exactly at the cutoff
    for dtype in (torch.float32, torch.float64):
        g = torch.Generator().manual_seed(21)
        pos = torch.rand((2000, 2), generator=g).to(dtype)
        pairs, order = capture_order(ns.cell_linked_pairs, pos, 0.05)
        data[f"c{k}_pos"], data[f"c{k}_cutoff"] = _np(pos), np.float64(0.05)
        data[f"c{k}_pairs"], data[f"c{k}_order"] = _np(pairs), _np(order)
        k += 1
        xs = torch.arange(20, dtype=dtype) * 0.1
        gx, gy = torch.meshgrid(xs, xs, indexing="xy")
        lat = torch.stack((gx.reshape(-1), gy.reshape(-1)), -1)
        pairs, order = capture_order(ns.cell_linked_pairs, lat, 0.2)
        data[f"c{k}_pos"], data[f"c{k}_cutoff"] = _np(lat), np.float64(0.2)
        data[f"c{k}_pairs"], data[f"c{k}_order"] = _np(pairs), _np(order)
        k += 1
    clustered = torch.full((30, 2), 2.5, dtype=torch.float64)
    clustered[0] = torch.tensor([-4.0, 7.0], dtype=torch.float64)
    pairs, order = capture_order(ns.cell_linked_pairs, clustered, 0.2)
    data[f"c{k}_pos"], data[f"c{k}_cutoff"] = _np(clustered), np.float64(0.2)
    data[f"c{k}_pairs"], data[f"c{k}_order"] = _np(pairs), _np(order)
    k += 1
    data["count"] = np.int64(k)
    return data


def periodic_cases(n3):
    data = {}
    k = 0
    for dtype in (torch.float32, torch.float64):
        for seed, npart, cutoff in ((7, 300, 0.12), (3, 800, 0.2)):
            g = torch.Generator().manual_seed(seed)
            pos = (torch.rand((npart, 3), generator=g)).to(dtype)
            pairs, order = capture_order(n3.periodic_pairs, pos, 1.0, cutoff)
            brute = n3.brute_force_pairs_min_image(pos, 1.0, cutoff)
            assert torch.equal(pairs, brute)
            data[f"c{k}_pos"], data[f"c{k}_cutoff"] = _np(pos), np.float64(cutoff)
            data[f"c{k}_box"] = np.float64(1.0)
            data[f"c{k}_pairs"], data[f"c{k}_order"] = _np(pairs), _np(order)
            k += 1
    data["count"] = np.int64(k)
    return data


def rhs2d_cases(di, db):
    """2-D ``rhs`` on dam-break states with walls, several option sets."""
    data = {}
    k = 0
    option_sets = [
        dict(),
        dict(density_diffusion=0.1),
        dict(density_diffusion=0.1, density_diffusion_form="antuono", wall_friction=0.5),
        dict(density_renormalization=True, wall_friction=1.0),
        dict(boundary_consistent_density=True),
    ]
    for dtype in (torch.float32, torch.float64):
        torch.set_default_dtype(dtype)
        try:
            for oi, opts in enumerate(option_sets):
                cfg = db.DamBreakConfig(dx=0.05, column_width=0.5, column_height=0.6,
                                        pool_width=1.2, tank_height=0.9, sound_speed=20.0,
                                        viscosity=1e-3, dt=2e-4, **opts)
                pos, mass = db.make_column(cfg, torch.device("cpu"))
                wall = di.wall_lattice(cfg, torch.device("cpu"), top=cfg.tank_top())
                g = torch.Generator().manual_seed(31 + oi)
                pos = pos + 0.1 * cfg.dx * torch.randn(pos.shape, generator=g).to(dtype)
                vel = 0.3 * torch.randn(pos.shape, generator=g).to(dtype)
                h = cfg.h_factor * cfg.dx
                all_pos = torch.cat((pos, wall))
                cache = di.PairListCache(2.0 * h, 0.25 * h, fluid_count=pos.shape[0])
                pairs, _ = cache.get(all_pos)
                split = oi in (2, 3)
                out = di.rhs(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt,
                             split=split)
                data[f"c{k}_pos"], data[f"c{k}_vel"] = _np(pos), _np(vel)
                data[f"c{k}_mass"], data[f"c{k}_wall"] = _np(mass), _np(wall)
                data[f"c{k}_pairs"] = _np(pairs)
                data[f"c{k}_opts"] = np.int64(oi)
                data[f"c{k}_split"] = np.int64(split)
                data[f"c{k}_rho"], data[f"c{k}_p"], data[f"c{k}_acc"] = map(_np, out[:3])
                if split:
                    data[f"c{k}_reaction"] = _np(out[3]["reaction"])
                    data[f"c{k}_face_pressure"] = _np(out[3]["face_pressure"])
                k += 1
        finally:
            torch.set_default_dtype(torch.float32)
    data["count"] = np.int64(k)
    return data


def config1_case(di, db):
    """One ``rhs`` of the 5,000-particle dam break (dx = 0.02) at rest."""
    data = {}
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 2.0)
    for tag, dtype in (("f32", torch.float32), ("f64", torch.float64)):
        torch.set_default_dtype(dtype)
        try:
            cfg = db.DamBreakConfig(dx=0.02, column_width=1.0, column_height=2.0,
                                    pool_width=4.0, tank_height=3.0, sound_speed=c0,
                                    viscosity=1e-6, max_courant=0.25,
                                    dt=0.25 * 1.3 * 0.02 / c0, steps=1000, wall_layers=3)
            pos, mass = db.make_column(cfg, torch.device("cpu"))
            wall = di.wall_lattice(cfg, torch.device("cpu"), top=cfg.tank_top())
            h = cfg.h_factor * cfg.dx
            cache = di.PairListCache(2.0 * h, cfg.pair_skin_factor * h,
                                     fluid_count=pos.shape[0])
            pairs, _ = cache.get(torch.cat((pos, wall)))
            vel = torch.zeros_like(pos)
            rho, p, acc = di.rhs(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt)
            # one semi-implicit Euler step and a second rhs from the moved state
            vel2 = vel + cfg.dt * acc
            pos2 = pos + cfg.dt * vel2
            di.apply_boundary(pos2, vel2, cfg, top=cfg.tank_top())
            pairs2, rebuilt = cache.get(torch.cat((pos2, wall)))
            rho2, p2, acc2 = di.rhs(pos2, vel2, mass, cfg, pairs=pairs2, wall=wall, dt=cfg.dt)
            for name, t in dict(pos=pos, mass=mass, wall=wall, pairs=pairs, rho=rho, p=p,
                                acc=acc, pos2=pos2, vel2=vel2, rho2=rho2, p2=p2,
                                acc2=acc2).items():
                data[f"{tag}_{name}"] = _np(t)
            data[f"{tag}_rebuilt2"] = np.int64(rebuilt)
        finally:
            torch.set_default_dtype(torch.float32)
    return data


def rhs3d_cases(d3, di):
    data = {}
    k = 0
    for dtype in (torch.float32, torch.float64):
        for opts in (dict(), dict(density_diffusion=0.1, wall_friction=0.3)):
            torch.set_default_dtype(dtype)
            try:
                cfg = d3.DamBreak3DConfig(dx=0.04, tank_height=0.4, tank_depth=0.2,
                                          column_width=0.2, column_depth=0.2,
                                          column_height=0.24, pool_width=0.5,
                                          sound_speed=15.0, viscosity=1e-3, dt=1e-4, **opts)
                pos, mass = d3.make_column_3d(cfg, torch.device("cpu"), seed=5)
                wall = d3.wall_lattice_3d(cfg, torch.device("cpu"))
                g = torch.Generator().manual_seed(9 + k)
                pos = pos + 0.1 * cfg.dx * torch.randn(pos.shape, generator=g).to(dtype)
                vel = 0.2 * torch.randn(pos.shape, generator=g).to(dtype)
                h = cfg.h_factor * cfg.dx
                cache = di.PairListCache(2.0 * h, 0.25 * h, fluid_count=pos.shape[0])
                pairs, _ = cache.get(torch.cat((pos, wall)))
                rho, p, acc, reaction = d3.rhs_3d(pos, vel, mass, cfg, pairs=pairs, wall=wall,
                                                  dt=cfg.dt, return_wall_force=True)
                for name, t in dict(pos=pos, vel=vel, mass=mass, wall=wall, pairs=pairs,
                                    rho=rho, p=p, acc=acc, reaction=reaction).items():
                    data[f"c{k}_{name}"] = _np(t)
                data[f"c{k}_diffusion"] = np.float64(cfg.density_diffusion)
                data[f"c{k}_friction"] = np.float64(cfg.wall_friction)
                k += 1
            finally:
                torch.set_default_dtype(torch.float32)
    data["count"] = np.int64(k)
    return data


def rhs3d_closure_cases(d3, di):
    """rhs_3d with the free-surface pressure closure (dam_break_3d.py:
    339-342) on jittered 3-D columns with walls, FP32 and FP64: "interior"
    donors with diffusion and friction, "all" donors."""
    data = {}
    k = 0
    for dtype in (torch.float32, torch.float64):
        for opts in (dict(surface_pressure_closure=True, density_diffusion=0.1, wall_friction=0.3),
                     dict(surface_pressure_closure=True, surface_pressure_donors="all")):
            torch.set_default_dtype(dtype)
            try:
                cfg = d3.DamBreak3DConfig(dx=0.04, tank_height=0.4, tank_depth=0.2,
                                          column_width=0.2, column_depth=0.2,
                                          column_height=0.24, pool_width=0.5,
                                          sound_speed=15.0, viscosity=1e-3, dt=1e-4, **opts)
                pos, mass = d3.make_column_3d(cfg, torch.device("cpu"), seed=5)
                wall = d3.wall_lattice_3d(cfg, torch.device("cpu"))
                g = torch.Generator().manual_seed(90 + k)
                pos = pos + 0.1 * cfg.dx * torch.randn(pos.shape, generator=g).to(dtype)
                vel = 0.2 * torch.randn(pos.shape, generator=g).to(dtype)
                h = cfg.h_factor * cfg.dx
                cache = di.PairListCache(2.0 * h, 0.25 * h, fluid_count=pos.shape[0])
                pairs, _ = cache.get(torch.cat((pos, wall)))
                rho, p, acc, reaction = d3.rhs_3d(pos, vel, mass, cfg, pairs=pairs, wall=wall,
                                                  dt=cfg.dt, return_wall_force=True)
                for name, t in dict(pos=pos, vel=vel, mass=mass, wall=wall, pairs=pairs,
                                    rho=rho, p=p, acc=acc, reaction=reaction).items():
                    data[f"c{k}_{name}"] = _np(t)
                data[f"c{k}_opts"] = np.array(repr(sorted(opts.items())))
                k += 1
            finally:
                torch.set_default_dtype(torch.float32)
    data["count"] = np.int64(k)
    return data


def threed_cases(t3):
    data = {}
    k = 0
    # periodic shear lattice with jitter (config 2 shape, reduced to 12^3)
    for dtype in (torch.float32, torch.float64):
        for order in (2, 4):
            n = 12
            dx = 1.0 / n
            h = 1.3 * dx
            pos = t3.cubic_lattice((n, n, n), dx, dtype=dtype)
            g = torch.Generator().manual_seed(3 + order)
            pos = (pos + (torch.rand(pos.shape, generator=g).to(dtype) - 0.5) * 0.02 * dx
                   ).remainder(1.0)
            mass = torch.full((pos.shape[0],), t3.calibrated_particle_mass(dx, h, 1000.0),
                              dtype=dtype)
            vel = torch.zeros_like(pos)
            vel[:, 0] = 1e-3 * torch.sin(2 * math.pi * pos[:, 2])
            pairs = t3.periodic_pairs(pos, 1.0, 2.5 * h)
            acc, rho, p = t3.accelerations(pos, vel, mass, h, pairs, rho0=1000.0,
                                           sound_speed=1.0, viscosity=1e-2, box=1.0,
                                           viscous_order=order)
            for name, t in dict(pos=pos, vel=vel, mass=mass, pairs=pairs, acc=acc,
                                rho=rho, p=p).items():
                data[f"c{k}_{name}"] = _np(t)
            data[f"c{k}_kind"] = np.int64(0)
            data[f"c{k}_h"], data[f"c{k}_order"] = np.float64(h), np.int64(order)
            k += 1
    # wall-bounded hydrostatic column with Antuono diffusion
    for dtype in (torch.float32, torch.float64):
        for form in ("antuono", "molteni"):
            dx = 0.01
            h = 1.3 * dx
            fluid = t3.cubic_lattice((6, 6, 5), dx, origin=(0.02, 0.02, 0.02), dtype=dtype)
            wall = t3.wall_shell((6, 6, 5), 2, dx, dtype=dtype)
            pos = torch.cat((fluid, wall))
            g = torch.Generator().manual_seed(17)
            pos[: fluid.shape[0]] += 0.05 * dx * torch.randn(fluid.shape, generator=g).to(dtype)
            mass = torch.full((pos.shape[0],), t3.calibrated_particle_mass(dx, h, 1000.0),
                              dtype=dtype)
            vel = 0.05 * torch.randn(pos.shape, generator=g).to(dtype)
            vel[fluid.shape[0]:] = 0
            pairs = t3.box_pairs(pos, 2.0 * h)
            acc, rho, p = t3.accelerations(
                pos, vel, mass, h, pairs, rho0=1000.0, sound_speed=20.0, viscosity=0.02,
                gravity=torch.tensor([0.0, 0.0, -9.81], dtype=dtype), n_fluid=fluid.shape[0],
                density_diffusion=0.1, dt=1e-4, density_diffusion_form=form)
            for name, t in dict(pos=pos, vel=vel, mass=mass, pairs=pairs, acc=acc,
                                rho=rho, p=p).items():
                data[f"c{k}_{name}"] = _np(t)
            data[f"c{k}_kind"] = np.int64(1 if form == "antuono" else 2)
            data[f"c{k}_h"], data[f"c{k}_nfluid"] = np.float64(h), np.int64(fluid.shape[0])
            k += 1
    data["count"] = np.int64(k)
    return data


def shift_cases(ps, di):
    data = {}
    k = 0
    for dtype in (torch.float32, torch.float64):
        for dim in (2, 3):
            g = torch.Generator().manual_seed(40 + dim)
            side = 14 if dim == 2 else 7
            dx = 0.05
            axes = [torch.arange(side, dtype=dtype) * dx for _ in range(dim)]
            grid = torch.stack(torch.meshgrid(*axes, indexing="ij"), -1).reshape(-1, dim)
            pos = grid + 0.15 * dx * torch.randn(grid.shape, generator=g).to(dtype)
            volume = torch.full((pos.shape[0],), dx ** dim, dtype=dtype) * (
                1.0 + 0.05 * torch.rand((pos.shape[0],), generator=g).to(dtype))
            h = 1.3 * dx
            out, state = ps.shift_positions(pos, volume, h, dt=1e-3, v_ref=2.0,
                                            return_state=True)
            for name, t in dict(pos=pos, volume=volume, out=out, c=state.concentration,
                                grad=state.grad_c, shift=state.shift).items():
                data[f"c{k}_{name}"] = _np(t)
            data[f"c{k}_h"], data[f"c{k}_cref"] = np.float64(h), np.float64(state.c_reference)
            k += 1
    data["count"] = np.int64(k)
    return data


def meters_cases(cons, di):
    """Conservation ledger rows (threed/conservation.py) and the pair-list
    density summation (droplet_impact.py:761-788) on seeded clouds."""
    data = {}
    k = 0
    for dtype in (torch.float32, torch.float64):
        for dim, box in ((3, None), (3, 0.5), (2, None)):
            g = torch.Generator().manual_seed(60 + k)
            n = 500
            pos = (0.5 * torch.rand((n, dim), generator=g)).to(dtype)
            vel = (0.1 * torch.randn((n, dim), generator=g)).to(dtype)
            mass = (1.0 + 0.1 * torch.rand((n,), generator=g)).to(dtype)
            rho = (1000.0 * (1.0 + 0.01 * torch.randn((n,), generator=g))).to(dtype)
            if dim == 3:
                row = cons.diagnostics(pos, vel, mass, rho, rho0=1000.0, sound_speed=20.0,
                                       gamma=7.0, periodic_box=box)
                for key in ("mass", "kinetic_energy", "internal_energy", "total_energy"):
                    data[f"c{k}_ledger_{key}"] = np.float64(row[key])
                for key in ("momentum", "angular_momentum", "centre_of_mass"):
                    data[f"c{k}_ledger_{key}"] = np.asarray(row[key], dtype=np.float64)
                data[f"c{k}_e"] = _np(cons.internal_energy(rho, 1000.0, 20.0, 7.0))
            data[f"c{k}_box"] = np.float64(-1.0 if box is None else box)
            h = 0.03
            pairs = di.cell_linked_pairs(pos, 2.0 * h)
            data[f"c{k}_rho_pairs"] = _np(di.density_from_neighbor_pairs(pos, mass, h, pairs))
            for name, t in dict(pos=pos, vel=vel, mass=mass, rho=rho).items():
                data[f"c{k}_{name}"] = _np(t)
            data[f"c{k}_dim"] = np.int64(dim)
            k += 1
    data["count"] = np.int64(k)
    return data


def shear_cases(sv):
    """Short runs of the reference double-shear decay (threed/solver.py:211)."""
    data = {}
    k = 0
    for dtype in (torch.float64, torch.float32):
        r = sv.run_shear_wave(n=12, steps=40, sample_every=10, dtype=dtype)
        data[f"c{k}_times"] = np.asarray(r.times, dtype=np.float64)
        data[f"c{k}_amplitudes"] = np.asarray(r.amplitudes, dtype=np.float64)
        data[f"c{k}_fit_rate"] = np.float64(r.fit_rate)
        data[f"c{k}_kinetic"] = np.asarray([d["kinetic_energy"] for d in r.diagnostics])
        data[f"c{k}_total"] = np.asarray([d["total_energy"] for d in r.diagnostics])
        data[f"c{k}_momentum"] = np.asarray([d["momentum"] for d in r.diagnostics])
        data[f"c{k}_pairs_last"] = np.int64(r.pairs_last)
        data[f"c{k}_rebuilds"] = np.int64(r.pair_rebuilds)
        data[f"c{k}_dtype"] = np.array(str(dtype))
        k += 1
    data["count"] = np.int64(k)
    return data


def csf_cases(ca, di):
    """Surface-tension acceleration and fields of the consistent CSF scheme
    (csf_consistent.py:384-446, fit_quadratic curvature) on a lattice drop, a
    jittered drop and a drop above a pool, and one full ``rhs`` with it."""
    data = {}
    k = 0
    for dtype in (torch.float64, torch.float32):
        for kind in ("drop", "jitter", "pool"):
            g = torch.Generator().manual_seed(80 + k)
            dx = 0.002
            h = 1.3 * dx
            if kind == "pool":
                cfg = di.Config(dx=dx, pool_width=0.08, pool_depth=0.02, drop_radius=0.01,
                                drop_center_y=0.035)
                pos, mass = di.make_particles(cfg, "cpu")
                pos, mass = pos.to(dtype), mass.to(dtype)
            else:
                ax = (torch.arange(-12, 13, dtype=torch.float64) * dx)
                gx, gy = torch.meshgrid(ax, ax, indexing="xy")
                pts = torch.stack((gx.reshape(-1), gy.reshape(-1)), -1)
                pts = pts[torch.linalg.vector_norm(pts, dim=1) <= 10.5 * dx]
                if kind == "jitter":
                    pts = pts + 0.05 * dx * torch.randn(pts.shape, generator=g, dtype=torch.float64)
                pos = (pts + 0.05).to(dtype)
                mass = torch.full((pos.shape[0],), 1000.0 * dx * dx, dtype=dtype)
            rho = (1000.0 * (1.0 + 0.002 * torch.randn((pos.shape[0],), generator=g,
                                                        dtype=torch.float64))).to(dtype)
            pairs = di.cell_linked_pairs(pos, 2.0 * h)
            acc, st = ca.surface_tension_acceleration(pos, rho, mass, pairs, h, 0.0728, rho0=1000.0,
                                                      curvature_scheme="fit_quadratic",
                                                      delta_normalization="legacy")
            for name, t in dict(pos=pos, mass=mass, rho=rho, acc=acc, color=st.color,
                                grad_c=st.grad_c, normal=st.normal, kappa=st.kappa,
                                delta_s=st.delta_s).items():
                data[f"c{k}_{name}"] = _np(t)
            data[f"c{k}_h"] = np.float64(h)
            k += 1
    data["count"] = np.int64(k)
    return data


def csf3_cases(c3, lc, ns, n3):
    """3-D CSF fields and acceleration (threed/csf3.py:113-238, "mls"
    curvature): a lattice ball, a jittered ball in FP64 and FP32, a jittered
    ball with a volume override and three stray particles (an isolated one
    and a close pair: degenerate MLS stencils), and the periodic
    Rayleigh-Plateau column of liquid_column.build_column in its box."""
    data = {}
    k = 0
    dx = 1.0e-3
    h = 1.3 * dx
    for dtype, kind in ((torch.float64, "ball"), (torch.float64, "jitter"), (torch.float32, "jitter"),
                        (torch.float64, "volume"), (torch.float64, "column")):
        g = torch.Generator().manual_seed(120 + k)
        box = None
        if kind == "column":
            cfg = lc.ColumnConfig(radius=4e-3, dx=dx, kR=0.6971, epsilon=0.02)
            pos, mass, box = lc.build_column(cfg)
            pos, mass = pos.to(dtype), mass.to(dtype)
            h = cfg.h
            pairs = n3.periodic_pairs(pos, box, 2.0 * h)
            box = [float(b) for b in box]
        else:
            ax = torch.arange(-7, 8, dtype=torch.float64) * dx
            gx, gy, gz = torch.meshgrid(ax, ax, ax, indexing="ij")
            pts = torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), -1)
            pts = pts[torch.linalg.vector_norm(pts, dim=1) <= 6.2 * dx]
            if kind != "ball":
                pts = pts + 0.08 * dx * torch.randn(pts.shape, generator=g, dtype=torch.float64)
            if kind == "volume":
                stray = torch.tensor([[0.03, 0.0, 0.0], [0.0, 0.03, 0.0], [0.0, 0.03 + dx, 0.0]],
                                     dtype=torch.float64)
                pts = torch.cat((pts, stray))
            pos = (pts + 0.02).to(dtype)
            mass = torch.full((pos.shape[0],), 1000.0 * dx ** 3, dtype=dtype)
            h = 1.3 * dx
            pairs = ns.cell_linked_pairs(pos, 2.0 * h)
        rho = (1000.0 * (1.0 + 0.002 * torch.randn((pos.shape[0],), generator=g,
                                                    dtype=torch.float64))).to(dtype)
        volume = (mass / rho) if kind == "volume" else None
        st = c3.csf_fields3(pos, mass, h, pairs, rho0=1000.0, box=box, volume=volume, curvature="mls")
        acc = c3.surface_tension_acceleration3(st, rho, 0.0728)
        fields = dict(pos=pos, mass=mass, rho=rho, pairs=pairs, acc=acc, color=st.color,
                      grad_c=st.grad_c, normal=st.normal, kappa=st.kappa, delta_s=st.delta_s,
                      valid=st.valid)
        if volume is not None:
            fields["volume"] = volume
        for name, t in fields.items():
            data[f"c{k}_{name}"] = _np(t)
        data[f"c{k}_h"] = np.float64(h)
        data[f"c{k}_box"] = np.asarray(box if box is not None else [0.0, 0.0, 0.0], dtype=np.float64)
        k += 1
    data["count"] = np.int64(k)
    return data


def csf3axi_cases(c3, lc, ns, n3):
    """The 3-D CSF with the "axisym" curvature (threed/csf3.py:159-220,
    meridional quadratic fit + n_r / r) on 4h pair lists: a jittered ball
    (FP64, FP32) and the periodic Rayleigh-Plateau column of
    liquid_column.build_column in its box (FP64)."""
    data = {}
    k = 0
    dx = 1.0e-3
    for dtype, kind in ((torch.float64, "ball"), (torch.float32, "ball"), (torch.float64, "column")):
        g = torch.Generator().manual_seed(500 + k)
        box = None
        if kind == "column":
            cfg = lc.ColumnConfig(radius=4e-3, dx=dx, kR=0.6971, epsilon=0.02)
            pos, mass, box = lc.build_column(cfg)
            pos, mass = pos.to(dtype), mass.to(dtype)
            h = cfg.h
            pairs = n3.periodic_pairs(pos, box, 4.0 * h)
            box = [float(b) for b in box]
        else:
            ax = torch.arange(-7, 8, dtype=torch.float64) * dx
            gx, gy, gz = torch.meshgrid(ax, ax, ax, indexing="ij")
            pts = torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), -1)
            pts = pts[torch.linalg.vector_norm(pts, dim=1) <= 6.2 * dx]
            pts = pts + 0.08 * dx * torch.randn(pts.shape, generator=g, dtype=torch.float64)
            pos = pts.to(dtype)
            mass = torch.full((pos.shape[0],), 1000.0 * dx ** 3, dtype=dtype)
            h = 1.3 * dx
            pairs = ns.cell_linked_pairs(pos, 4.0 * h)
        rho = (1000.0 * (1.0 + 0.002 * torch.randn((pos.shape[0],), generator=g,
                                                    dtype=torch.float64))).to(dtype)
        st = c3.csf_fields3(pos, mass, h, pairs, rho0=1000.0, box=box, curvature="axisym")
        acc = c3.surface_tension_acceleration3(st, rho, 0.0728)
        fields = dict(pos=pos, mass=mass, rho=rho, pairs=pairs, acc=acc, color=st.color,
                      grad_c=st.grad_c, normal=st.normal, kappa=st.kappa, delta_s=st.delta_s,
                      valid=st.valid)
        for name, t in fields.items():
            data[f"c{k}_{name}"] = _np(t)
        data[f"c{k}_h"] = np.float64(h)
        data[f"c{k}_box"] = np.asarray(box if box is not None else [0.0, 0.0, 0.0], dtype=np.float64)
        k += 1
    data["count"] = np.int64(k)
    return data


def tvc_cases(tv, ns):
    """transport_velocity_correction (transport_velocity_correction.py:285-513)
    on jittered fluid blocks with wall layers: 2-D and 3-D, FP64 and FP32, no
    limiter and TruncatedLinear, with max_shift, an active scope, scope_tol and
    a per-particle h_ratio."""
    data = {}
    opts = [
        ("2d", torch.float64, dict()),
        ("2d", torch.float32, dict()),
        ("2d", torch.float64, dict(limiter="tl", max_shift=2e-5, scope_tol=0.5)),
        ("2d", torch.float64, dict(active=True, alpha=0.2, h_ref=0.0031)),
        ("2d", torch.float64, dict(h_ratio=True)),
        ("3d", torch.float64, dict()),
        ("3d", torch.float64, dict(limiter="tl")),
    ]
    for k, (kind, dtype, o) in enumerate(opts):
        g = torch.Generator().manual_seed(200 + k)
        dx = 0.002
        h = 1.3 * dx
        dim = 2 if kind == "2d" else 3
        nx = 14 if dim == 2 else 8
        ax = torch.arange(nx, dtype=torch.float64) * dx + 0.5 * dx
        grids = torch.meshgrid(*([ax] * dim), indexing="ij")
        fluid = torch.stack([t.reshape(-1) for t in grids], -1)
        fluid = fluid + 0.08 * dx * torch.randn(fluid.shape, generator=g, dtype=torch.float64)
        # three wall layers under the block (y < 0)
        wl = torch.arange(-3, 0, dtype=torch.float64) * dx + 0.5 * dx
        wx = torch.arange(-3, nx + 3, dtype=torch.float64) * dx + 0.5 * dx
        if dim == 2:
            WX, WY = torch.meshgrid(wx, wl, indexing="ij")
            wall = torch.stack((WX.reshape(-1), WY.reshape(-1)), -1)
        else:
            WX, WY, WZ = torch.meshgrid(wx, wl, wx, indexing="ij")
            wall = torch.stack((WX.reshape(-1), WY.reshape(-1), WZ.reshape(-1)), -1)
        pos = torch.cat((fluid, wall)).to(dtype)
        nf, nw = fluid.shape[0], wall.shape[0]
        volume = (dx ** dim * (1.0 + 0.01 * torch.randn(pos.shape[0], generator=g,
                                                       dtype=torch.float64))).to(dtype)
        kw = dict(wall_count=nw)
        search_h = h
        if o.get("h_ratio"):
            ratio = (1.0 + 0.3 * torch.rand(nf, generator=g, dtype=torch.float64)).to(dtype)
            ratio[::7] = 0.8
            kw["h_ratio"] = ratio
            search_h = h / 0.8
        pairs = ns.cell_linked_pairs(pos, 2.0 * search_h)
        if o.get("limiter") == "tl":
            kw["limiter"] = tv.truncated_linear(100.0)
        for name in ("max_shift", "scope_tol", "alpha", "h_ref"):
            if name in o:
                kw[name] = o[name]
        if o.get("active"):
            kw["active"] = torch.arange(nf) % 3 != 0
        res = tv.transport_velocity_correction(pos, volume, h, pairs=pairs, **kw)
        data[f"c{k}_pos"] = _np(pos)
        data[f"c{k}_volume"] = _np(volume)
        data[f"c{k}_pairs"] = _np(pairs)
        data[f"c{k}_h"] = np.float64(h)
        data[f"c{k}_n_wall"] = np.int64(nw)
        data[f"c{k}_opts"] = np.array(repr(sorted((a, b) for a, b in o.items())))
        for name in ("max_shift", "scope_tol", "alpha", "h_ref"):
            if name in o:
                data[f"c{k}_{name}"] = np.float64(o[name])
        data[f"c{k}_limiter_tl"] = np.int64(o.get("limiter") == "tl")
        if o.get("active"):
            data[f"c{k}_active"] = _np(kw["active"])
        if o.get("h_ratio"):
            data[f"c{k}_h_ratio"] = _np(kw["h_ratio"])
        for name in ("gradient_integral", "shift", "squared_norm", "limiter"):
            data[f"c{k}_{name}"] = _np(getattr(res, name))
        data[f"c{k}_clipped"] = np.float64(res.clipped)
    data["count"] = np.int64(len(opts))
    return data


def csf2d_cases(ca, di):
    """2-D CSF variants (csf_consistent.py:262-446): curvature "mls",
    "fit_quadratic" and "fit_circle", delta_s "legacy" and "local_range", normal smoothing off,
    curvature from a smoothed colour field, FP64 and FP32, through
    surface_tension_acceleration (the 4h list for the fit) and through direct
    csf_fields calls on a 2h list (the smoothing options are csf_fields
    arguments only)."""
    data = {}
    variants = [
        ("jitter", torch.float64, dict(curvature_scheme="mls")),
        ("jitter", torch.float64, dict(curvature_scheme="mls", delta_normalization="local_range")),
        ("pool", torch.float64, dict(curvature_scheme="fit_quadratic", delta_normalization="local_range")),
        ("jitter", torch.float64, dict(curvature_scheme="mls", curvature_color_smoothing=1, direct=True)),
        ("jitter", torch.float64, dict(curvature_scheme="mls", normal_smoothing=0, direct=True)),
        ("jitter", torch.float32, dict(curvature_scheme="fit_quadratic")),
        ("jitter", torch.float64, dict(curvature_scheme="fit_quadratic", direct=True)),
        ("pool", torch.float64, dict(curvature_scheme="fit_circle")),
        ("jitter", torch.float64, dict(curvature_scheme="fit_circle", delta_normalization="local_range")),
        ("jitter", torch.float32, dict(curvature_scheme="fit_circle")),
        ("jitter", torch.float64, dict(curvature_scheme="fit_circle", direct=True)),
    ]
    for k, (kind, dtype, o) in enumerate(variants):
        g = torch.Generator().manual_seed(300 + k)
        dx = 0.002
        h = 1.3 * dx
        if kind == "pool":
            cfg = di.Config(dx=dx, pool_width=0.08, pool_depth=0.02, drop_radius=0.01, drop_center_y=0.035)
            pos, mass = di.make_particles(cfg, "cpu")
            pos, mass = pos.to(dtype), mass.to(dtype)
        else:
            ax = torch.arange(-12, 13, dtype=torch.float64) * dx
            gx, gy = torch.meshgrid(ax, ax, indexing="xy")
            pts = torch.stack((gx.reshape(-1), gy.reshape(-1)), -1)
            pts = pts[torch.linalg.vector_norm(pts, dim=1) <= 10.5 * dx]
            pts = pts + 0.05 * dx * torch.randn(pts.shape, generator=g, dtype=torch.float64)
            pos = (pts + 0.05).to(dtype)
            mass = torch.full((pos.shape[0],), 1000.0 * dx * dx, dtype=dtype)
        rho = (1000.0 * (1.0 + 0.002 * torch.randn((pos.shape[0],), generator=g, dtype=torch.float64))).to(dtype)
        o = dict(o)
        direct = o.pop("direct", False)
        pairs = di.cell_linked_pairs(pos, 2.0 * h)
        if direct:
            st = ca.csf_fields(pos, mass, pairs, h, 1000.0, **o)
            acc = None
        else:
            acc, st = ca.surface_tension_acceleration(pos, rho, mass, pairs, h, 0.0728, rho0=1000.0, **o)
        fields = dict(pos=pos, mass=mass, rho=rho, pairs=pairs, color=st.color, grad_c=st.grad_c,
                      normal=st.normal, kappa=st.kappa, delta_s=st.delta_s)
        if acc is not None:
            fields["acc"] = acc
        for name, t in fields.items():
            data[f"c{k}_{name}"] = _np(t)
        data[f"c{k}_h"] = np.float64(h)
        data[f"c{k}_direct"] = np.int64(direct)
        data[f"c{k}_opts"] = np.array(repr(sorted(o.items())))
    data["count"] = np.int64(len(variants))
    return data


def contact_cases(ca, seed=400):
    """The contact-angle terms of the 2-D CSF (csf_consistent.py:411-560,
    contact_angle_isph.py:75-213) on a jittered sessile half-drop (radius
    10 dx) on a flat three-layer wall lattice: nearest_wall (one particle
    sitting on a wall particle), apply_contact_angle_boundary at two angles,
    and csf_fields / surface_tension_acceleration with the "rotate" boundary
    and the "young" and "brackbill" tractions, FP64 and FP32."""
    data = {}
    dx = 0.002
    h = 1.3 * dx
    wx = torch.arange(-16, 17, dtype=torch.float64) * dx
    wall64 = torch.cat([torch.stack((wx, torch.full_like(wx, -0.5 * dx - k * dx)), -1) for k in range(3)])
    ax = (torch.arange(-11, 11, dtype=torch.float64) + 0.5) * dx
    gx, gy = torch.meshgrid(ax, (torch.arange(0, 11, dtype=torch.float64) + 0.5) * dx, indexing="xy")
    pts = torch.stack((gx.reshape(-1), gy.reshape(-1)), -1)
    pts = pts[torch.linalg.vector_norm(pts, dim=1) <= 10.5 * dx]
    g = torch.Generator().manual_seed(seed)
    pts64 = pts + 0.05 * dx * torch.randn(pts.shape, generator=g, dtype=torch.float64)
    rho64 = 1000.0 * (1.0 + 0.002 * torch.randn((pts.shape[0],), generator=g, dtype=torch.float64))
    grad64 = torch.randn(pts.shape, generator=g, dtype=torch.float64) * 100.0
    # standalone nearest_wall with one particle on a wall particle, and the boundary
    probe = torch.cat((pts64, wall64[40:41]))
    d, nrm = ca.nearest_wall(probe, wall64)
    data.update(nw_pos=_np(probe), nw_dist=_np(d), nw_normal=_np(nrm), wall=_np(wall64), h=np.float64(h))
    for k, theta in enumerate((math.pi / 6, 2 * math.pi / 3)):
        data[f"bc{k}_theta"] = np.float64(theta)
        data[f"bc{k}_out"] = _np(ca.apply_contact_angle_boundary(grad64.clone(), pts64, wall64, h, theta))
    data["bc_grad"] = _np(grad64)
    variants = [
        (torch.float64, dict(contact_angle=math.pi / 3, contact_angle_model="rotate", curvature_scheme="mls")),
        (torch.float64, dict(contact_angle=2 * math.pi / 3, contact_angle_model="rotate",
                             curvature_scheme="fit_quadratic")),
        (torch.float64, dict(contact_angle=math.pi / 3, curvature_color_smoothing=1, direct=True)),
        (torch.float64, dict(contact_angle=math.pi / 3, contact_angle_model="young", curvature_scheme="mls")),
        (torch.float64, dict(contact_angle=2 * math.pi / 3, contact_angle_model="brackbill",
                             curvature_scheme="fit_quadratic")),
        (torch.float32, dict(contact_angle=math.pi / 3, contact_angle_model="rotate", curvature_scheme="mls")),
        (torch.float32, dict(contact_angle=math.pi / 3, contact_angle_model="young", curvature_scheme="mls")),
    ]
    from tensorsph.neighbor_search import cell_linked_pairs
    for k, (dtype, o) in enumerate(variants):
        pos, wall, rho = pts64.to(dtype), wall64.to(dtype), rho64.to(dtype)
        mass = torch.full((pos.shape[0],), 1000.0 * dx * dx, dtype=dtype)
        pairs = cell_linked_pairs(pos, 2.0 * h)
        o = dict(o)
        direct = o.pop("direct", False)
        if direct:
            st = ca.csf_fields(pos, mass, pairs, h, 1000.0, wall=wall, **o)
            acc = None
        else:
            acc, st = ca.surface_tension_acceleration(pos, rho, mass, pairs, h, 0.0728, rho0=1000.0, wall=wall, **o)
        fields = dict(pos=pos, mass=mass, rho=rho, pairs=pairs, color=st.color, grad_c=st.grad_c,
                      normal=st.normal, kappa=st.kappa, delta_s=st.delta_s)
        if acc is not None:
            fields["acc"] = acc
        for name, t in fields.items():
            data[f"c{k}_{name}"] = _np(t)
        data[f"c{k}_direct"] = np.int64(direct)
        data[f"c{k}_opts"] = np.array(repr(sorted(o.items())))
    data["count"] = np.int64(len(variants))
    return data


def rhs_csf_cases(di):
    """droplet_impact.rhs with CSF surface tension (droplet_impact.py:1210-1222:
    the fluid pairs of the step's list through compute_surface_tension_force)
    on a jittered drop above a walled pool, FP64 (default dtype float64, so
    the wall masses are not rounded to FP32): the default options, "mls" with
    "local_range", and contact angles with "rotate" and "young"."""
    saved = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        return _rhs_csf_cases(di)
    finally:
        torch.set_default_dtype(saved)


def _rhs_csf_cases(di):
    data = {}
    dx = 0.002
    variants = [dict(), dict(csf_curvature="mls", csf_delta_normalization="local_range"),
                dict(contact_angle=math.pi / 3),
                dict(contact_angle=2 * math.pi / 3, contact_angle_model="young")]
    for k, o in enumerate(variants):
        cfg = di.Config(dx=dx, pool_width=0.08, pool_depth=0.02, drop_radius=0.01, drop_center_y=0.035,
                        surface_tension_coefficient=0.0728, density_diffusion=0.1, **o)
        pos, mass = di.make_particles(cfg, "cpu")
        wall = di.wall_lattice(cfg, "cpu").double()
        g = torch.Generator().manual_seed(600 + k)
        pos = pos.double() + 0.02 * dx * torch.randn(pos.shape, generator=g, dtype=torch.float64)
        mass = mass.double()
        vel = 0.01 * torch.randn(pos.shape, generator=g, dtype=torch.float64)
        h = cfg.h_factor * cfg.dx
        pairs = di.cell_linked_pairs(torch.cat((pos, wall)), 2.0 * h)
        rho, p, acc = di.rhs(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt)
        for name, t in dict(pos=pos, vel=vel, mass=mass, wall=wall, pairs=pairs, rho=rho, p=p,
                            acc=acc).items():
            data[f"c{k}_{name}"] = _np(t)
        data[f"c{k}_opts"] = np.array(repr(sorted(o.items())))
    data["count"] = np.int64(len(variants))
    return data


def dt_cases(di):
    """The step-limit helpers (droplet_impact.py:495-556, surface_tension.py:
    294-318) on a few configurations and speeds."""
    rows = []
    for o in (dict(), dict(viscosity=1e-3), dict(density_diffusion=0.1, surface_tension_coefficient=0.0728),
              dict(dt_growth=0.9, surface_tension_coefficient=0.5, dx=0.001)):
        cfg = di.Config(**o)
        from tensorsph.surface_tension import capillary_dt_limit
        for speed in (0.0, 1.5, 30.0):
            for dt in (cfg.dt, 0.5 * cfg.dt):
                rows.append([di.acoustic_dt_limit(cfg, speed), capillary_dt_limit(cfg), di.stable_dt(cfg, speed),
                             di.next_dt(cfg, dt, speed)])
    return {"values": np.asarray(rows, dtype=np.float64)}


def dense_cases(di):
    """rhs_all_pairs (droplet_impact.py:1232-1281), the dense O(N^2)
    formulation without walls, on seeded jittered blocks in FP64: plain, with
    Molteni diffusion, with the "antuono" form selected (the dense
    formulation keeps the Molteni term), with viscosity, and with the
    free-surface pressure closure ("interior" and "all" donors, whose dense
    pair set holds each particle with itself)."""
    data = {}
    variants = [dict(), dict(density_diffusion=0.1), dict(density_diffusion=0.1, density_diffusion_form="antuono"),
                dict(viscosity=1e-3, density_diffusion=0.05),
                dict(surface_pressure_closure=True, density_diffusion=0.05),
                dict(surface_pressure_closure=True, surface_pressure_donors="all")]
    for k, o in enumerate(variants):
        g = torch.Generator().manual_seed(700 + k)
        dx = 0.02
        cfg = di.Config(dx=dx, pool_width=0.4, pool_depth=0.15, drop_radius=0.05, drop_center_y=0.25, **o)
        ax = (torch.arange(0, 14, dtype=torch.float64) + 0.5) * dx
        gx, gy = torch.meshgrid(ax, ax, indexing="xy")
        pos = torch.stack((gx.reshape(-1), gy.reshape(-1)), -1)
        pos = pos + 0.1 * dx * torch.randn(pos.shape, generator=g, dtype=torch.float64)
        vel = 0.05 * torch.randn(pos.shape, generator=g, dtype=torch.float64)
        mass = torch.full((pos.shape[0],), 1000.0 * dx * dx, dtype=torch.float64)
        rho, p, acc = di.rhs_all_pairs(pos, vel, mass, cfg)
        for name, t in dict(pos=pos, vel=vel, mass=mass, rho=rho, p=p, acc=acc).items():
            data[f"c{k}_{name}"] = _np(t)
        data[f"c{k}_opts"] = np.array(repr(sorted(o.items())))
    data["count"] = np.int64(len(variants))
    return data


def delta_plus_cases(dp):
    """delta_plus_step on a perturbed lattice block in a walled corner (fluid,
    slip walls with normals, gravity, diffusion) and on a free block."""
    data = {}
    k = 0
    for dtype in (torch.float64, torch.float32):
        for kind in ("tank", "free"):
            g = torch.Generator().manual_seed(90 + k)
            dx = 0.01
            ax = (torch.arange(12, dtype=torch.float64) + 0.5) * dx
            pos = torch.cartesian_prod(ax, ax)
            pos = pos + 0.08 * dx * torch.randn(pos.shape, generator=g, dtype=torch.float64)
            vel = 0.05 * torch.randn(pos.shape, generator=g, dtype=torch.float64)
            rho = 1000.0 + 2.0 * torch.randn((pos.shape[0],), generator=g, dtype=torch.float64)
            mass = torch.full((pos.shape[0],), 1000.0 * dx * dx, dtype=torch.float64)
            kw = dict(dx=dx, sound_speed=20.0, reference_speed=0.5, dt=1e-4, gravity=9.81,
                      viscosity=1e-6, diffusion=0.1, alpha=0.02)
            wall = wall_v = wall_n = None
            if kind == "tank":
                # three rows of stations below the floor y = 0 and left of x = 0
                layers = []
                normals = []
                xs = (torch.arange(-3, 16, dtype=torch.float64) + 0.5) * dx
                for m in range(1, 4):
                    ys = torch.full_like(xs, (0.5 - m) * dx)
                    layers.append(torch.stack((xs, ys), 1))
                    normals.append(torch.tensor([[0.0, 1.0]]).expand(xs.numel(), 2))
                    yy = (torch.arange(0, 16, dtype=torch.float64) + 0.5) * dx
                    layers.append(torch.stack((torch.full_like(yy, (0.5 - m) * dx), yy), 1))
                    normals.append(torch.tensor([[1.0, 0.0]]).expand(yy.numel(), 2))
                wall = torch.cat(layers).to(dtype)
                wall_n = torch.cat(normals).to(dtype).contiguous()
                wall_v = torch.zeros_like(wall)
            st = dp.delta_plus_step(pos.to(dtype), vel.to(dtype), rho.to(dtype), mass.to(dtype),
                                    wall=wall, wall_velocity=wall_v, wall_normal=wall_n, **kw)
            for name, t in dict(pos=pos.to(dtype), vel=vel.to(dtype), rho=rho.to(dtype),
                                mass=mass.to(dtype), out_position=st.position,
                                out_velocity=st.velocity, out_density=st.density,
                                out_acceleration=st.acceleration, out_wall_reaction=st.wall_reaction,
                                out_shift=st.shift).items():
                data[f"c{k}_{name}"] = _np(t)
            if wall is not None:
                data[f"c{k}_wall"] = _np(wall)
                data[f"c{k}_wall_normal"] = _np(wall_n)
            k += 1
    data["count"] = np.int64(k)
    return data


def config1_run_case(db):
    """The reference's own 2-D dam-break loop (dam_break.run_case) on the
    5,000-particle configuration for 150 steps in FP64: sampled front and
    energies and the final positions."""
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 2.0)
    torch.set_default_dtype(torch.float64)
    try:
        cfg = db.DamBreakConfig(dx=0.02, column_width=1.0, column_height=2.0, pool_width=4.0,
                                tank_height=3.0, sound_speed=c0, viscosity=1e-6, max_courant=0.25,
                                dt=0.25 * 1.3 * 0.02 / c0, steps=150, output_every=50,
                                wall_layers=3, device="cpu")
        run = db.run_case(cfg)
    finally:
        torch.set_default_dtype(torch.float32)
    return {"times": np.asarray(run.times), "front": np.asarray(run.front),
            "kinetic": np.asarray(run.kinetic_energy), "potential": np.asarray(run.potential_energy),
            "final_positions": _np(run.final_positions), "rebuilds": np.int64(run.rebuilds),
            "escaped": np.int64(run.escaped), "steps": np.int64(run.steps_taken)}


def dam3d_run_case(d3):
    """The reference's own 3-D dam-break loop (dam_break_3d.run_case) on a
    small tank for 40 steps in FP64, with Molteni diffusion and wall friction."""
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 0.24)
    torch.set_default_dtype(torch.float64)
    try:
        cfg = d3.DamBreak3DConfig(dx=0.02, pool_width=0.5, tank_depth=0.2, tank_height=0.4,
                                  column_width=0.2, column_depth=0.2, column_height=0.24,
                                  sound_speed=c0, viscosity=1e-3, dt=0.25 * 1.3 * 0.02 / c0,
                                  density_diffusion=0.1, wall_friction=0.3, steps=40,
                                  output_every=10, device="cpu")
        run = d3.run_case(cfg)
    finally:
        torch.set_default_dtype(torch.float32)
    return {"times": np.asarray(run.times), "front": np.asarray(run.front),
            "kinetic": np.asarray(run.kinetic_energy), "potential": np.asarray(run.potential_energy),
            "final_positions": _np(run.final_positions), "rebuilds": np.int64(run.rebuilds),
            "escaped": np.int64(run.escaped), "steps": np.int64(run.steps_taken),
            "max_speed": np.float64(run.max_speed),
            "max_density_compression": np.float64(run.max_density_compression)}


REGULARIZED_OPTION_SETS = [
    dict(density_regularization="compression"),
    dict(density_regularization="compression", compression_regularization_rule="internal",
         compression_normalization="none", wall_friction=0.5),
    dict(surface_pressure_closure=True, density_diffusion=0.1),
    dict(surface_pressure_closure=True, surface_pressure_donors="all"),
    dict(surface_pressure_closure=True, surface_pressure_layers=3, boundary_consistent_density=True),
]


def regularized_cases(di, db):
    """2-D ``rhs`` with the compression density regularisation
    (droplet_impact.py:982-1028, two calls sharing one ``state``: the second
    uses the inverse reference compression the first wrote) and the
    free-surface pressure closure (:1030-1037, 429-492) on jittered resting
    columns with walls, FP32 and FP64."""
    data = {}
    k = 0
    for dtype in (torch.float32, torch.float64):
        torch.set_default_dtype(dtype)
        try:
            for oi, opts in enumerate(REGULARIZED_OPTION_SETS):
                cfg = db.DamBreakConfig(dx=0.05, column_width=0.5, column_height=0.6,
                                        pool_width=1.2, tank_height=0.9, sound_speed=20.0,
                                        viscosity=1e-3, dt=2e-4, **opts)
                pos, mass = db.make_column(cfg, torch.device("cpu"))
                wall = di.wall_lattice(cfg, torch.device("cpu"), top=cfg.tank_top())
                g = torch.Generator().manual_seed(61 + oi)
                pos = pos + 0.1 * cfg.dx * torch.randn(pos.shape, generator=g).to(dtype)
                vel = 0.3 * torch.randn(pos.shape, generator=g).to(dtype)
                h = cfg.h_factor * cfg.dx
                cache = di.PairListCache(2.0 * h, 0.25 * h, fluid_count=pos.shape[0])
                pairs, _ = cache.get(torch.cat((pos, wall)))
                state = {}
                for call in (0, 1):
                    out = di.rhs(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt, state=state)
                    data[f"c{k}_rho{call}"], data[f"c{k}_p{call}"], data[f"c{k}_acc{call}"] = map(_np, out[:3])
                    if "compression" in state:
                        data[f"c{k}_kref{call}"] = np.float64(state["compression"].inverse_reference_compression)
                        data[f"c{k}_counted{call}"] = np.int64(state["compression_counted"])
                data[f"c{k}_pos"], data[f"c{k}_vel"] = _np(pos), _np(vel)
                data[f"c{k}_mass"], data[f"c{k}_wall"] = _np(mass), _np(wall)
                data[f"c{k}_pairs"] = _np(pairs)
                data[f"c{k}_opts"] = np.int64(oi)
                k += 1
        finally:
            torch.set_default_dtype(torch.float32)
    data["count"] = np.int64(k)
    return data


def adaptive_run_case(db):
    """The reference's own 2-D dam-break loop with adaptive_dt (dam_break.py:
    362-465) in FP64 on the tank of its Courant-limit test (dx = 0.04,
    c0 = 25, 0.25 s): the step-size range, the Courant peak, the sampled
    meters and the final positions."""
    torch.set_default_dtype(torch.float64)
    try:
        cfg = db.DamBreakConfig(dx=0.04, pool_width=2.0, column_width=0.2, column_height=0.4,
                                sound_speed=25.0, adaptive_dt=True, device="cpu")
        cfg.dt = cfg.dt_from_courant()
        cfg.steps = int(round(0.25 / cfg.dt))
        cfg.output_every = max(1, int(round(0.05 / cfg.dt)))
        run = db.run_case(cfg)
    finally:
        torch.set_default_dtype(torch.float32)
    return {"times": np.asarray(run.times), "front": np.asarray(run.front),
            "kinetic": np.asarray(run.kinetic_energy), "potential": np.asarray(run.potential_energy),
            "final_positions": _np(run.final_positions), "rebuilds": np.int64(run.rebuilds),
            "escaped": np.int64(run.escaped), "steps": np.int64(run.steps_taken),
            "simulated_time": np.float64(run.simulated_time), "dt_min": np.float64(run.dt_min),
            "dt_max": np.float64(run.dt_max), "max_acoustic_courant": np.float64(run.max_acoustic_courant),
            "max_speed": np.float64(run.max_speed), "dt": np.float64(cfg.dt),
            "cfg_steps": np.int64(cfg.steps), "output_every": np.int64(cfg.output_every)}


def checkpoint_case(kl):
    """A checkpoint file as the obstacle case writes it (save_checkpoint,
    kleefsman_obstacle_3d.py:499-528): its bytes, the configuration's
    fingerprint and the inputs, for the format tests."""
    import json
    import tempfile
    cfg = kl.Kleefsman3DConfig(dx=0.05)
    g = torch.Generator().manual_seed(300)
    pos = torch.rand((12, 3), generator=g, dtype=torch.float64)
    vel = torch.randn((12, 3), generator=g, dtype=torch.float64)
    run = kl.Kleefsman3DRun(cfg=cfg, fluid_particles=12, wall_particles=5)
    run.times, run.slab, run.local_h2 = [0.0, 0.0065], [0.01, 0.02], [0.011, 0.021]
    run.height, run.front, run.bypass = [0.012, 0.022], [1.2, 1.3], [0.0, 1.0]
    run.sph_impulse, run.clamp_impulse = [0.5, -0.25, 0.125], [0.0, 0.03125, 0.0]
    args = dict(step=25, elapsed=0.0065, dt=2.6e-4, speeds=1.5, compression=0.01, escapes=2, clamps=1)
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "state.pt"
        kl.save_checkpoint(path, cfg, positions=pos, velocity=vel, run=run, **args)
        raw = path.read_bytes()
    series = {k: getattr(run, k) for k in ("times", "slab", "local_h2", "height", "front", "bypass",
                                           "sph_impulse", "clamp_impulse")}
    return {"raw": np.frombuffer(raw, dtype=np.uint8).copy(),
            "fingerprint": np.array(json.dumps(kl.checkpoint_fingerprint(cfg))),
            "fields": np.array(json.dumps(list(kl.CHECKPOINT_FINGERPRINT_FIELDS))),
            "version": np.array(kl.CHECKPOINT_VERSION),
            "args": np.array(json.dumps(args)), "series": np.array(json.dumps(series)),
            "pos": _np(pos), "vel": _np(vel)}


HYDROSTATIC_CASES = [
    dict(nx=6, ny=5, nz=7, steps=30, sample_every=5, settle_fraction=0.5),
    dict(nx=5, ny=5, nz=6, steps=24, sample_every=4, settle_fraction=0.5, lid=False,
         density_diffusion=0.1, wall_model="adami"),
]


def hydrostatic_cases(sv):
    """Short runs of the reference's wall-bounded column (threed/solver.py:353-484):
    the sampled bottom pressure and centre of mass, and the profile's rows,
    lattice rows and scalar accuracy numbers."""
    data = {}
    for k, kw in enumerate(HYDROSTATIC_CASES):
        r = sv.run_hydrostatic(dtype=torch.float64, **kw)
        prof = r.profile
        data[f"c{k}_times"] = np.asarray(r.times, dtype=np.float64)
        data[f"c{k}_bottom"] = np.asarray(r.bottom_pressure, dtype=np.float64)
        data[f"c{k}_com"] = np.asarray(r.centre_of_mass_z, dtype=np.float64)
        data[f"c{k}_counts"] = np.asarray([r.steps, r.fluid_particles, r.wall_particles], dtype=np.int64)
        data[f"c{k}_rows_p"] = np.asarray([row["p_measured"] for row in prof["rows"]], dtype=np.float64)
        data[f"c{k}_rows_rho"] = np.asarray([row["rho_measured"] for row in prof["rows"]], dtype=np.float64)
        data[f"c{k}_lat_p"] = np.asarray([row["p_measured"] for row in prof["rows_by_lattice"]], dtype=np.float64)
        data[f"c{k}_lat_z"] = np.asarray([row["z"] for row in prof["rows_by_lattice"]], dtype=np.float64)
        for key in ("integral_p_measured", "odd_even_amplitude_over_scale", "max_rel_error_core_lattice",
                    "wall_displacement"):
            data[f"c{k}_{key}"] = np.float64(prof[key] if prof[key] is not None else np.nan)
        data[f"c{k}_binning"] = np.asarray([prof["binning"][key] for key in
                                            ("mean_offset_over_dx", "rms_offset_over_dx", "misplaced_fraction")])
        data[f"c{k}_kinetic"] = np.float64(r.diagnostics[0]["kinetic_energy"])
    data["count"] = np.int64(len(HYDROSTATIC_CASES))
    return data


def main(src, families=None):
    sys.path.insert(0, str(src))
    import tensorsph.neighbor_search as ns
    import tensorsph.droplet_impact as di
    import tensorsph.dam_break as db
    import tensorsph.dam_break_3d as d3
    import tensorsph.particle_shifting as ps
    import tensorsph.threed as t3
    from tensorsph.threed import neighbors3 as n3
    from tensorsph.threed import conservation as cons
    from tensorsph.threed import solver as sv
    import tensorsph.csf_consistent as ca
    import tensorsph.delta_plus as dp
    from tensorsph.threed import csf3 as c3
    from tensorsph.threed import liquid_column as lc
    import tensorsph.transport_velocity_correction as tv
    import tensorsph.kleefsman_obstacle_3d as kl

    meta = {"torch_version": np.array(torch.__version__)}
    torch.set_num_threads(1)
    makers = {
        "pairs": lambda: pairs_cases(ns),
        "periodic": lambda: periodic_cases(n3),
        "rhs2d": lambda: rhs2d_cases(di, db),
        "config1": lambda: config1_case(di, db),
        "rhs3d": lambda: rhs3d_cases(d3, di),
        "threed": lambda: threed_cases(t3),
        "shift": lambda: shift_cases(ps, di),
        "meters": lambda: meters_cases(cons, di),
        "shear": lambda: shear_cases(sv),
        "csf": lambda: csf_cases(ca, di),
        "delta_plus": lambda: delta_plus_cases(dp),
        "csf3": lambda: csf3_cases(c3, lc, ns, n3),
        "tvc": lambda: tvc_cases(tv, ns),
        "csf2d": lambda: csf2d_cases(ca, di),
        "config1_run": lambda: config1_run_case(db),
        "dam3d_run": lambda: dam3d_run_case(d3),
        "checkpoint": lambda: checkpoint_case(kl),
        "contact": lambda: contact_cases(ca),
        "csf3axi": lambda: csf3axi_cases(c3, lc, ns, n3),
        "rhs_csf": lambda: rhs_csf_cases(di),
        "dense": lambda: dense_cases(di),
        "dt": lambda: dt_cases(di),
        "adaptive_run": lambda: adaptive_run_case(db),
        "regularized": lambda: regularized_cases(di, db),
        "rhs3d_closure": lambda: rhs3d_closure_cases(d3, di),
        "hydrostatic": lambda: hydrostatic_cases(sv),
    }
    for name in families or makers:
        np.savez_compressed(OUT / f"{name}.npz", **makers[name](), **meta)


RHS2D_OPTION_SETS = [
    dict(),
    dict(density_diffusion=0.1),
    dict(density_diffusion=0.1, density_diffusion_form="antuono", wall_friction=0.5),
    dict(density_renormalization=True, wall_friction=1.0),
    dict(boundary_consistent_density=True),
]

if __name__ == "__main__":
    # make_golden.py SRC [FAMILY ...]: regenerate the named families (default all)
    # from the reference source tree SRC (the directory that holds `tensorsph/`)
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py SRC [FAMILY ...]  (SRC: the reference's src/ directory)")
    main(Path(sys.argv[1]), sys.argv[2:] or None)
