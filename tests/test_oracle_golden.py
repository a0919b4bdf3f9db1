"""Pin the numpy oracle against fixtures produced by the reference itself."""
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import neighbors as on
from oracle import pairpass as op
from tests.golden.make_golden import RHS2D_OPTION_SETS


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) / scale


def test_pairs_and_cell_order_bit_exact(golden):
    g = golden("pairs")
    for k in range(int(g["count"])):
        pos, cutoff = g[f"c{k}_pos"], float(g[f"c{k}_cutoff"])
        pairs = on.cell_linked_pairs(pos, cutoff)
        assert np.array_equal(pairs, g[f"c{k}_pairs"]), k
        *_, order = on.cell_grid(pos, cutoff)
        assert np.array_equal(order, g[f"c{k}_order"]), k
        assert np.array_equal(on.cell_linked_pairs_batched(pos, cutoff), g[f"c{k}_pairs"]), k
        if pos.shape[0] <= 400:
            assert np.array_equal(on.brute_force_pairs(pos, cutoff), g[f"c{k}_pairs"]), k


def test_periodic_pairs_bit_exact(golden):
    g = golden("periodic")
    for k in range(int(g["count"])):
        pos, cutoff = g[f"c{k}_pos"], float(g[f"c{k}_cutoff"])
        pairs = on.periodic_pairs(pos, float(g[f"c{k}_box"]), cutoff)
        assert np.array_equal(pairs, g[f"c{k}_pairs"]), k
        *_, order = on.periodic_grid(pos, float(g[f"c{k}_box"]), cutoff)
        assert np.array_equal(order, g[f"c{k}_order"]), k


def _cfg2d(opts, **kw):
    base = dict(dx=0.05, h_factor=1.3, rho0=1000.0, sound_speed=20.0, gamma=7.0,
                gravity=9.81, viscosity=1e-3, dt=2e-4, wall_friction=0.0,
                density_diffusion=0.0, density_diffusion_form="molteni",
                density_diffusion_eigenvalue_floor=0.1, density_calibration=True,
                density_renormalization=False, boundary_consistent_density=False)
    base.update(kw)
    base.update(opts)
    return SimpleNamespace(**base)


def test_rhs2d_matches_reference(golden):
    g = golden("rhs2d")
    for k in range(int(g["count"])):
        opts = RHS2D_OPTION_SETS[int(g[f"c{k}_opts"])]
        cfg = _cfg2d(opts)
        split = bool(g[f"c{k}_split"])
        out = op.rhs(g[f"c{k}_pos"], g[f"c{k}_vel"], g[f"c{k}_mass"], cfg,
                     pairs=g[f"c{k}_pairs"], wall=g[f"c{k}_wall"], dt=cfg.dt, split=split)
        tol = 1e-12 if g[f"c{k}_pos"].dtype == np.float64 else 2e-5
        assert rel_err(out[0], g[f"c{k}_rho"]) < tol, k
        assert rel_err(out[1], g[f"c{k}_p"]) < max(tol, 1e-11) * 50, k
        assert rel_err(out[2], g[f"c{k}_acc"]) < max(tol, 1e-11) * 50, k
        if split:
            assert rel_err(out[3]["reaction"], g[f"c{k}_reaction"]) < max(tol, 1e-11) * 50
            assert rel_err(out[3]["face_pressure"], g[f"c{k}_face_pressure"]) < max(tol, 1e-11) * 50


def test_config1_state_matches_reference(golden):
    import math
    g = golden("config1")
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 2.0)
    cfg = _cfg2d({}, dx=0.02, sound_speed=c0, viscosity=1e-6, dt=0.25 * 1.3 * 0.02 / c0)
    for tag in ("f32", "f64"):
        pos = g[f"{tag}_pos"]
        rho, p, acc = op.rhs(pos, np.zeros_like(pos), g[f"{tag}_mass"], cfg,
                             pairs=g[f"{tag}_pairs"], wall=g[f"{tag}_wall"], dt=cfg.dt)
        tol = 1e-12 if tag == "f64" else 2e-5
        assert rel_err(rho, g[f"{tag}_rho"]) < tol
        assert rel_err(p, g[f"{tag}_p"]) < tol * 50
        assert rel_err(acc, g[f"{tag}_acc"]) < tol * 50


def test_rhs3d_matches_reference(golden):
    g = golden("rhs3d")
    for k in range(int(g["count"])):
        cfg = SimpleNamespace(dx=0.04, h_factor=1.3, rho0=1000.0, sound_speed=15.0, gamma=7.0,
                              gravity=9.81, viscosity=1e-3, dt=1e-4,
                              wall_friction=float(g[f"c{k}_friction"]),
                              density_diffusion=float(g[f"c{k}_diffusion"]),
                              density_diffusion_form="molteni", density_calibration=True)
        out = op.rhs_3d(g[f"c{k}_pos"], g[f"c{k}_vel"], g[f"c{k}_mass"], cfg,
                        pairs=g[f"c{k}_pairs"], wall=g[f"c{k}_wall"], dt=cfg.dt,
                        return_wall_force=True)
        tol = 1e-12 if g[f"c{k}_pos"].dtype == np.float64 else 2e-5
        for got, name in zip(out, ("rho", "p", "acc", "reaction")):
            assert rel_err(got, g[f"c{k}_{name}"]) < tol * (1 if name == "rho" else 50), (k, name)


def test_threed_accelerations_match_reference(golden):
    g = golden("threed")
    for k in range(int(g["count"])):
        kind = int(g[f"c{k}_kind"])
        pos = g[f"c{k}_pos"]
        tol = 1e-12 if pos.dtype == np.float64 else 2e-5
        if kind == 0:
            acc, rho, p = op.accelerations(pos, g[f"c{k}_vel"], g[f"c{k}_mass"],
                                           float(g[f"c{k}_h"]), g[f"c{k}_pairs"],
                                           rho0=1000.0, sound_speed=1.0, viscosity=1e-2,
                                           box=1.0, viscous_order=int(g[f"c{k}_order"]))
        else:
            acc, rho, p = op.accelerations(
                pos, g[f"c{k}_vel"], g[f"c{k}_mass"], float(g[f"c{k}_h"]), g[f"c{k}_pairs"],
                rho0=1000.0, sound_speed=20.0, viscosity=0.02,
                gravity=np.array([0.0, 0.0, -9.81]), n_fluid=int(g[f"c{k}_nfluid"]),
                density_diffusion=0.1, dt=1e-4,
                density_diffusion_form="antuono" if kind == 1 else "molteni")
        assert rel_err(rho, g[f"c{k}_rho"]) < tol, k
        assert rel_err(p, g[f"c{k}_p"]) < tol * 1e3, k
        assert rel_err(acc, g[f"c{k}_acc"]) < tol * 1e3, k


def test_shift_positions_match_reference(golden):
    g = golden("shift")
    for k in range(int(g["count"])):
        pos = g[f"c{k}_pos"]
        out, st = op.shift_positions(pos, g[f"c{k}_volume"], float(g[f"c{k}_h"]),
                                     dt=1e-3, v_ref=2.0)
        tol = 1e-12 if pos.dtype == np.float64 else 2e-5
        assert rel_err(st["concentration"], g[f"c{k}_c"]) < tol
        assert rel_err(st["grad_c"], g[f"c{k}_grad"]) < tol * 100
        assert abs(st["c_reference"] - float(g[f"c{k}_cref"])) <= 1e-6 * abs(float(g[f"c{k}_cref"]))
        assert rel_err(st["shift"], g[f"c{k}_shift"]) < tol * 100
        assert rel_err(out - pos, g[f"c{k}_out"] - pos) < tol * 1e3


def test_pair_cache_rebuild_rule():
    rng = np.random.default_rng(3)
    pos = rng.random((200, 2))
    cache = on.PairListCache(0.1, 0.02, fluid_count=150)
    p1, rebuilt = cache.get(pos)
    assert rebuilt and cache.rebuilds == 1
    _, rebuilt = cache.get(pos + 0.006)  # |d| = 0.0085 < skin / 2
    assert not rebuilt and cache.reuses == 1
    _, rebuilt = cache.get(pos + 0.02)
    assert rebuilt and cache.rebuilds == 2
    assert ((p1[:, 0] < 150) | (p1[:, 1] < 150)).all()
    with pytest.raises(ValueError):
        on.PairListCache(0.0, 0.1)


def test_meters_oracle_matches_reference(golden):
    """The oracle's conservation ledger and pair-list density against the
    reference's own outputs (threed/conservation.py, droplet_impact.py:761)."""
    from oracle import meters as om
    from oracle.neighbors import cell_linked_pairs
    g = golden("meters")
    for k in range(int(g["count"])):
        pos, vel, mass, rho = (g[f"c{k}_{n}"] for n in ("pos", "vel", "mass", "rho"))
        fp32 = pos.dtype == np.float32
        box = float(g[f"c{k}_box"])
        if int(g[f"c{k}_dim"]) == 3:
            row = om.diagnostics(pos, vel, mass, rho, rho0=1000.0, sound_speed=20.0, gamma=7.0,
                                 periodic_box=None if box < 0 else box)
            tol = 2e-6 if fp32 else 1e-12
            for key in ("mass", "kinetic_energy", "momentum", "angular_momentum", "centre_of_mass"):
                ref = np.asarray(g[f"c{k}_ledger_{key}"])
                assert np.abs(np.asarray(row[key]) - ref).max() <= tol * max(np.abs(ref).max(), 1.0), (k, key)
            # the internal energy is quadratic in (rho - rho0): a relative
            # comparison against a sum of small terms
            ie = float(g[f"c{k}_ledger_internal_energy"])
            assert abs(row["internal_energy"] - ie) <= (5e-3 if fp32 else 1e-9) * abs(ie), k
            e = om.internal_energy(rho, 1000.0, 20.0, 7.0)
            assert np.abs(e - g[f"c{k}_e"]).max() <= (2e-2 if fp32 else 1e-9) * np.abs(g[f"c{k}_e"]).max()
        pairs = cell_linked_pairs(pos, 0.06)
        dens = om.density_from_neighbor_pairs(pos, mass, 0.03, pairs)
        ref = g[f"c{k}_rho_pairs"]
        assert np.abs(dens - ref).max() <= (2e-6 if fp32 else 1e-12) * np.abs(ref).max(), k


def test_csf_oracle_matches_reference(golden):
    """The oracle's consistent CSF (fit_quadratic curvature) against the
    reference's own FP64 output; fields compared where they carry force
    (delta_s > 0: interior normals are round-off directions)."""
    from oracle import csf
    g = golden("csf")
    for k in range(int(g["count"])):
        pos = g[f"c{k}_pos"]
        if pos.dtype != np.float64:
            continue
        acc, st = csf.surface_tension_acceleration(pos, g[f"c{k}_rho"], g[f"c{k}_mass"],
                                                   float(g[f"c{k}_h"]), 0.0728, 1000.0)
        ref = g[f"c{k}_acc"]
        assert np.abs(acc - ref).max() <= 1e-10 * np.abs(ref).max(), k
        live = g[f"c{k}_delta_s"] > 0
        for name in ("color", "grad_c", "delta_s"):
            r = g[f"c{k}_{name}"]
            assert np.abs(st[name] - r).max() <= 1e-12 * max(np.abs(r).max(), 1.0), (k, name)
        for name in ("normal", "kappa"):
            r = g[f"c{k}_{name}"][live]
            assert np.abs(st[name][live] - r).max() <= 1e-8 * np.abs(r).max(), (k, name)


def _csf3_case(g, k):
    box = g[f"c{k}_box"]
    return dict(pos=g[f"c{k}_pos"], mass=g[f"c{k}_mass"], rho=g[f"c{k}_rho"], pairs=g[f"c{k}_pairs"],
                h=float(g[f"c{k}_h"]), box=box if box.any() else None,
                volume=g.get(f"c{k}_volume"))


def test_csf3_oracle_matches_reference(golden):
    """The oracle's 3-D CSF ("mls") against the reference's own output
    (tests/golden/csf3.npz).  The perfect lattice ball (case 0) is
    ill-conditioned -- its interior |grad c| is round-off, so interior
    normals, and the curvature of their neighbours, follow the noise -- and
    is compared on the acceleration only."""
    from oracle import csf3
    g = golden("csf3")
    for k in range(int(g["count"])):
        c = _csf3_case(g, k)
        st = csf3.csf_fields3(c["pos"], c["mass"], c["h"], c["pairs"], rho0=1000.0, box=c["box"],
                              volume=c["volume"])
        acc = csf3.surface_tension_acceleration3(st, c["rho"], 0.0728)
        f64 = c["pos"].dtype == np.float64
        ref = g[f"c{k}_acc"]
        assert np.abs(acc - ref).max() <= (1e-4 if k == 0 else (1e-12 if f64 else 1e-5)) * np.abs(ref).max(), k
        if k == 0:
            continue
        assert (st["valid"] == g[f"c{k}_valid"]).all(), k
        tol = 1e-12 if f64 else 1e-5
        for name in ("color", "grad_c", "delta_s", "normal", "kappa"):
            r = g[f"c{k}_{name}"]
            assert np.abs(st[name] - r).max() <= tol * max(np.abs(r).max(), 1.0), (k, name)


def _tvc_kwargs(g, k):
    kw = dict(wall_count=int(g[f"c{k}_n_wall"]))
    for name in ("max_shift", "scope_tol", "alpha", "h_ref"):
        if f"c{k}_{name}" in g:
            kw[name] = float(g[f"c{k}_{name}"])
    if f"c{k}_active" in g:
        kw["active"] = g[f"c{k}_active"]
    if f"c{k}_h_ratio" in g:
        kw["h_ratio"] = g[f"c{k}_h_ratio"]
    return kw


def test_csf2d_oracle_variants_match_reference(golden):
    """The oracle's 2-D CSF variants (mls / fit_quadratic curvature, legacy /
    local_range delta_s, normal smoothing off, smoothed-colour curvature)
    against the reference's own output (tests/golden/csf2d.npz)."""
    import ast
    from oracle import csf
    g = golden("csf2d")
    for k in range(int(g["count"])):
        o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
        pos, mass, rho, pairs, h = (g[f"c{k}_pos"], g[f"c{k}_mass"], g[f"c{k}_rho"], g[f"c{k}_pairs"],
                                    float(g[f"c{k}_h"]))
        if int(g[f"c{k}_direct"]):
            st = csf.csf_fields(pos, mass, pairs, h, 1000.0, **o)
        else:
            acc, st = csf.surface_tension_acceleration(pos, rho, mass, h, 0.0728, 1000.0, pairs=pairs, **o)
            ref = g[f"c{k}_acc"]
            assert np.abs(acc - ref).max() <= (1e-10 if pos.dtype == np.float64 else 1e-4) * np.abs(ref).max()
        live = g[f"c{k}_delta_s"] > 0
        tol = 1e-9 if pos.dtype == np.float64 else 1e-4
        for name in ("color", "grad_c", "delta_s", "normal", "kappa"):
            r, d = g[f"c{k}_{name}"], st[name]
            if name in ("normal", "kappa"):
                r, d = r[live], d[live]
            assert np.abs(d - r).max() <= tol * max(np.abs(r).max(), 1.0), (k, name)


def test_tvc_oracle_matches_reference(golden):
    """The oracle's transport-velocity correction against the reference's own
    output (tests/golden/tvc.npz: 2-D and 3-D, FP64 and FP32, limiters,
    max_shift, active scope, scope_tol, per-particle h_ratio)."""
    from oracle import tvc
    g = golden("tvc")
    for k in range(int(g["count"])):
        kw = _tvc_kwargs(g, k)
        if int(g[f"c{k}_limiter_tl"]):
            kw["slope"] = 100.0
        pos = g[f"c{k}_pos"]
        r = tvc.transport_velocity_correction(pos, g[f"c{k}_volume"], float(g[f"c{k}_h"]), g[f"c{k}_pairs"], **kw)
        tol = 1e-13 if pos.dtype == np.float64 else 2e-6
        for name in ("gradient_integral", "shift", "squared_norm", "limiter"):
            ref = g[f"c{k}_{name}"]
            assert np.abs(r[name] - ref).max() <= tol * np.abs(ref).max(), (k, name)
        assert r["clipped"] == float(g[f"c{k}_clipped"]), k


def test_delta_plus_oracle_matches_reference(golden):
    """The oracle's delta-plus step against the reference's own output
    (tests/golden/delta_plus.npz: a walled corner and a free block)."""
    from oracle import delta_plus as odp
    g = golden("delta_plus")
    kw = dict(dx=0.01, sound_speed=20.0, reference_speed=0.5, dt=1e-4, gravity=9.81, viscosity=1e-6,
              diffusion=0.1, alpha=0.02)
    for k in range(int(g["count"])):
        wall = g[f"c{k}_wall"] if f"c{k}_wall" in g else None
        wn = g[f"c{k}_wall_normal"] if wall is not None else None
        out = odp.delta_plus_step(g[f"c{k}_pos"], g[f"c{k}_vel"], g[f"c{k}_rho"], g[f"c{k}_mass"],
                                  wall=wall, wall_normal=wn, **kw)
        tol = 1e-12 if g[f"c{k}_pos"].dtype == np.float64 else 5e-6
        for key in ("position", "velocity", "density", "acceleration", "wall_reaction", "shift"):
            ref = g[f"c{k}_out_{key}"]
            if ref.size:
                assert np.abs(out[key] - ref).max() <= tol * np.abs(ref).max(), (k, key)


def _contact_compare(st, acc, g, k, f64, tol_dir):
    live = g[f"c{k}_delta_s"] > 0
    tol = 1e-9 if f64 else 1e-4
    for name in ("color", "grad_c", "delta_s"):
        r = g[f"c{k}_{name}"]
        assert np.abs(st[name] - r).max() <= tol * max(np.abs(r).max(), 1.0), (k, name)
    for name in ("normal", "kappa"):
        r = g[f"c{k}_{name}"][live]
        assert np.abs(st[name][live] - r).max() <= tol_dir * np.abs(r).max(), (k, name)
    if acc is not None:
        r = g[f"c{k}_acc"]
        assert np.abs(acc - r).max() <= tol_dir * np.abs(r).max(), (k, "acc")


def test_contact_angle_oracle_matches_reference(golden):
    """nearest_wall, apply_contact_angle_boundary and the CSF with the
    "rotate" boundary and the "young" / "brackbill" tractions against the
    reference's own outputs (tests/golden/contact.npz)."""
    import ast
    from oracle import contact_angle as oc
    from oracle import csf
    g = golden("contact")
    wall, h = g["wall"], float(g["h"])
    d, nrm = oc.nearest_wall(g["nw_pos"], wall)
    assert np.abs(d - g["nw_dist"]).max() <= 1e-12
    assert np.abs(nrm - g["nw_normal"]).max() <= 1e-12
    pos = g["nw_pos"][:-1]
    for k in range(2):
        out = oc.apply_contact_angle_boundary(g["bc_grad"], pos, wall, h, float(g[f"bc{k}_theta"]))
        assert np.abs(out - g[f"bc{k}_out"]).max() <= 1e-12 * np.abs(g[f"bc{k}_out"]).max()
    for k in range(int(g["count"])):
        o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
        p, mass, rho, pairs = g[f"c{k}_pos"], g[f"c{k}_mass"], g[f"c{k}_rho"], g[f"c{k}_pairs"]
        w = wall.astype(p.dtype)
        f64 = p.dtype == np.float64
        if int(g[f"c{k}_direct"]):
            st = csf.csf_fields(p, mass, pairs, h, 1000.0, stencil=4.0, curvature_scheme="mls", wall=w,
                                contact_angle=o["contact_angle"],
                                curvature_color_smoothing=o.get("curvature_color_smoothing", 0))
            acc = None
        else:
            acc, st = csf.surface_tension_acceleration(p, rho, mass, h, 0.0728, 1000.0, pairs=pairs, wall=w,
                                                       curvature_scheme=o["curvature_scheme"],
                                                       contact_angle=o["contact_angle"],
                                                       contact_angle_model=o["contact_angle_model"])
        _contact_compare(st, acc, g, k, f64, 1e-8 if f64 else 1e-3)


def test_csf3_axisym_oracle_matches_reference(golden):
    """The oracle's 3-D CSF with the "axisym" curvature (meridional quadratic
    fit + n_r / r) against the reference's own output
    (tests/golden/csf3axi.npz): FP64 within 1e-9 of the largest curvature,
    FP32 within 1e-3."""
    from oracle import csf3
    g = golden("csf3axi")
    for k in range(int(g["count"])):
        pos = g[f"c{k}_pos"]
        box = g[f"c{k}_box"]
        st = csf3.csf_fields3(pos, g[f"c{k}_mass"], float(g[f"c{k}_h"]), g[f"c{k}_pairs"], rho0=1000.0,
                              box=None if not box.any() else box, curvature="axisym")
        tol = 1e-9 if pos.dtype == np.float64 else 1e-3
        live = g[f"c{k}_delta_s"] > 1e-3 * g[f"c{k}_delta_s"].max()
        r = g[f"c{k}_kappa"][live]
        assert np.abs(st["kappa"][live] - r).max() <= tol * np.abs(r).max(), k
        acc = csf3.surface_tension_acceleration3(st, g[f"c{k}_rho"], 0.0728)
        ra = g[f"c{k}_acc"]
        assert np.abs(acc - ra).max() <= tol * np.abs(ra).max(), k


def test_rhs_with_csf_oracle_matches_reference(golden):
    """The droplet rhs with CSF surface tension (droplet_impact.py:1210-1222)
    as the oracle's rhs plus its CSF over the fluid pairs, against the
    reference's own rhs (tests/golden/rhs_csf.npz): default options, "mls" +
    "local_range", contact angles "rotate" and "young"."""
    import ast
    from dataclasses import replace
    from oracle import csf
    from oracle import pairpass as op
    from tensorsph_b200.droplet_impact import Config
    g = golden("rhs_csf")
    for k in range(int(g["count"])):
        o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
        cfg = replace(Config(dx=0.002, pool_width=0.08, pool_depth=0.02, drop_radius=0.01, drop_center_y=0.035,
                             surface_tension_coefficient=0.0728, density_diffusion=0.1), **o)
        pos, vel, mass, wall, pairs = (g[f"c{k}_{n}"] for n in ("pos", "vel", "mass", "wall", "pairs"))
        h = cfg.h_factor * cfg.dx
        plain = replace(cfg, surface_tension_coefficient=0.0)
        rho, p, acc = op.rhs(pos, vel, mass, plain, pairs=pairs, wall=wall, dt=cfg.dt)
        n = pos.shape[0]
        fluid = pairs[(pairs[:, 0] < n) & (pairs[:, 1] < n)]
        a_st, _ = csf.surface_tension_acceleration(
            pos, rho, mass, h, cfg.surface_tension_coefficient, cfg.rho0, pairs=fluid,
            curvature_scheme=cfg.csf_curvature, delta_normalization=cfg.csf_delta_normalization, wall=wall,
            contact_angle=cfg.contact_angle, contact_angle_model=cfg.contact_angle_model)
        assert np.abs(rho - g[f"c{k}_rho"]).max() <= 1e-12 * cfg.rho0
        ref = g[f"c{k}_acc"]
        assert np.abs(acc + a_st - ref).max() <= 1e-9 * np.abs(a_st).max(), k


REGULARIZED_DEFAULTS = dict(density_regularization="none", compression_regularization_rule="free_surface",
                            compression_normalization="reference_mean", surface_pressure_closure=False,
                            surface_pressure_threshold=0.99, surface_pressure_donors="interior",
                            surface_pressure_layers=2)


def test_regularized_rhs_matches_reference(golden):
    """The oracle's compression regularisation and free-surface closure
    against the reference's rhs (tests/golden/regularized.npz): two calls
    sharing one state, the written inverse reference compression and count."""
    from tests.golden.make_golden import REGULARIZED_OPTION_SETS
    g = golden("regularized")
    for k in range(int(g["count"])):
        opts = {**REGULARIZED_DEFAULTS, **REGULARIZED_OPTION_SETS[int(g[f"c{k}_opts"])]}
        cfg = _cfg2d(opts)
        tol = 1e-12 if g[f"c{k}_pos"].dtype == np.float64 else 2e-5
        state = {}
        for call in (0, 1):
            out = op.rhs(g[f"c{k}_pos"], g[f"c{k}_vel"], g[f"c{k}_mass"], cfg, pairs=g[f"c{k}_pairs"],
                         wall=g[f"c{k}_wall"], dt=cfg.dt, state=state)
            assert rel_err(out[0], g[f"c{k}_rho{call}"]) < tol, (k, call)
            assert rel_err(out[1], g[f"c{k}_p{call}"]) < max(tol, 1e-11) * 50, (k, call)
            assert rel_err(out[2], g[f"c{k}_acc{call}"]) < max(tol, 1e-11) * 50, (k, call)
            if f"c{k}_kref{call}" in g:
                assert state["inverse_reference"] == pytest.approx(float(g[f"c{k}_kref{call}"]), rel=tol)
                assert state["counted"] == int(g[f"c{k}_counted{call}"])


def test_rhs3d_closure_matches_reference(golden):
    """The oracle's rhs_3d with the free-surface closure against the
    reference's (tests/golden/rhs3d_closure.npz)."""
    import ast
    g = golden("rhs3d_closure")
    for k in range(int(g["count"])):
        opts = {**REGULARIZED_DEFAULTS, "wall_friction": 0.0, "density_diffusion": 0.0,
                **dict(ast.literal_eval(str(g[f"c{k}_opts"])))}
        cfg = SimpleNamespace(dx=0.04, h_factor=1.3, rho0=1000.0, sound_speed=15.0, gamma=7.0, gravity=9.81,
                              viscosity=1e-3, dt=1e-4, density_diffusion_form="molteni", density_calibration=True,
                              **opts)
        out = op.rhs_3d(g[f"c{k}_pos"], g[f"c{k}_vel"], g[f"c{k}_mass"], cfg, pairs=g[f"c{k}_pairs"],
                        wall=g[f"c{k}_wall"], dt=cfg.dt, return_wall_force=True)
        tol = 1e-12 if g[f"c{k}_pos"].dtype == np.float64 else 2e-5
        for got, name in zip(out, ("rho", "p", "acc", "reaction")):
            assert rel_err(got, g[f"c{k}_{name}"]) < tol * (1 if name == "rho" else 50), (k, name)
