"""GPU parity of the WCSPH pair pass with the reference (fixtures) and the oracle.

Tolerances, all max-norm:
* density: |d rho| / max|rho| < 1e-12 (FP64), 1e-5 (FP32);
* pressure: |d p| / B < 1e-12 (FP64), 1e-5 (FP32), with B = rho0 c0^2 / gamma the
  Tait bulk modulus -- near rho0 the EOS turns a density round-off e into
  gamma B e, so max|p| is the wrong yardstick;
* acceleration and wall reaction: |d a| / max|a| < 1e-11 (FP64), 1e-4 (FP32);
  in FP32 the hydrostatic balance cancels pressure terms ~1e3 times larger
  than the net acceleration (measured: 6.8e-5 on the 5,000-particle dam break,
  where the reference's own FP32 run is 6.1e-4 away from its FP64 run).
Fixtures were produced with torch's default dtype equal to the case dtype
(the reference rounds the wall mass to the default dtype), so each case runs
under the same default.
"""
import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import pairpass as op
from tests.golden.make_golden import RHS2D_OPTION_SETS

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float64): (1e-12, 1e-11), np.dtype(np.float32): (1e-5, 1e-4)}


def rel_err(a, b, scale=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = scale if scale is not None else max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) / s


def bulk(cfg):
    return cfg.rho0 * cfg.sound_speed ** 2 / cfg.gamma


@pytest.fixture
def default_dtype():
    saved = torch.get_default_dtype()
    yield torch.set_default_dtype
    torch.set_default_dtype(saved)


def _cfg(**kw):
    from tensorsph_b200.droplet_impact import Config
    return Config(**kw)


def test_rhs2d_matches_reference(gpu, golden, default_dtype):
    from tensorsph_b200.droplet_impact import rhs
    g = golden("rhs2d")
    for k in range(int(g["count"])):
        default_dtype(torch.from_numpy(g[f"c{k}_pos"][:1]).dtype)
        opts = RHS2D_OPTION_SETS[int(g[f"c{k}_opts"])]
        cfg = _cfg(dx=0.05, sound_speed=20.0, viscosity=1e-3, dt=2e-4, **opts)
        t = {name: torch.from_numpy(g[f"c{k}_{name}"]).to(gpu)
             for name in ("pos", "vel", "mass", "wall", "pairs")}
        split = bool(g[f"c{k}_split"])
        out = rhs(t["pos"], t["vel"], t["mass"], cfg, pairs=t["pairs"], wall=t["wall"],
                  dt=cfg.dt, split=split)
        tr, tf = TOL[g[f"c{k}_pos"].dtype]
        assert rel_err(out[0].cpu(), g[f"c{k}_rho"]) < tr, (k, "rho")
        assert rel_err(out[1].cpu(), g[f"c{k}_p"], bulk(cfg)) < tr, (k, "p")
        assert rel_err(out[2].cpu(), g[f"c{k}_acc"]) < tf, (k, "acc")
        if split:
            assert rel_err(out[3]["reaction"].cpu(), g[f"c{k}_reaction"]) < tf, (k, "reaction")
            assert rel_err(out[3]["face_pressure"].cpu(), g[f"c{k}_face_pressure"]) < tf


def test_config1_dam_break_state(gpu, golden, default_dtype):
    """One rhs of the 5,000-particle dam break at dx = 0.02, FP32 and FP64."""
    from tensorsph_b200.droplet_impact import rhs
    from tensorsph_b200.neighbor_search import PairListCache
    g = golden("config1")
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 2.0)
    cfg = _cfg(dx=0.02, sound_speed=c0, viscosity=1e-6, max_courant=0.25,
               dt=0.25 * 1.3 * 0.02 / c0, wall_layers=3)
    for tag in ("f32", "f64"):
        default_dtype(torch.float32 if tag == "f32" else torch.float64)
        pos = torch.from_numpy(g[f"{tag}_pos"]).to(gpu)
        wall = torch.from_numpy(g[f"{tag}_wall"]).to(gpu)
        mass = torch.from_numpy(g[f"{tag}_mass"]).to(gpu)
        h = cfg.h_factor * cfg.dx
        cache = PairListCache(2.0 * h, 0.25 * h, fluid_count=pos.shape[0])
        pairs, _ = cache.get(torch.cat((pos, wall)))
        assert np.array_equal(pairs.cpu().numpy(), g[f"{tag}_pairs"])
        rho, p, acc = rhs(pos, torch.zeros_like(pos), mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt)
        tr, tf = TOL[g[f"{tag}_pos"].dtype]
        assert rel_err(rho.cpu(), g[f"{tag}_rho"]) < tr
        assert rel_err(p.cpu(), g[f"{tag}_p"], bulk(cfg)) < tr
        assert rel_err(acc.cpu(), g[f"{tag}_acc"]) < tf


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rhs2d_optional_inputs_match_oracle(gpu, dtype, default_dtype):
    """nu_field, wall_vel, wall_accel, wrap_width and density_offset against the oracle."""
    from tensorsph_b200.droplet_impact import rhs, wall_lattice
    default_dtype(torch.float32 if dtype == np.float32 else torch.float64)
    cfg = _cfg(dx=0.05, pool_width=1.0, pool_depth=0.4, drop_radius=0.05, drop_center_y=0.6,
               sound_speed=20.0, viscosity=1e-3, dt=2e-4, wall_friction=0.7,
               density_diffusion=0.1)
    rng = np.random.default_rng(12)
    xs = (np.arange(20) + 0.5) * cfg.dx
    ys = (np.arange(8) + 0.5) * cfg.dx
    gx, gy = np.meshgrid(xs, ys, indexing="xy")
    pos = np.stack((gx.ravel(), gy.ravel()), -1).astype(dtype)
    pos = pos + (0.1 * cfg.dx * rng.standard_normal(pos.shape)).astype(dtype)
    n = pos.shape[0]
    vel = (0.2 * rng.standard_normal(pos.shape)).astype(dtype)
    mass = np.full(n, 2.4, dtype=dtype)
    wall = wall_lattice(cfg, "cpu", top=0.6).numpy().astype(dtype)
    nw = wall.shape[0]
    nu = (1e-3 * (1 + rng.random(n))).astype(dtype)
    wv = (0.1 * rng.standard_normal((nw, 2))).astype(dtype)
    wa = (0.5 * rng.standard_normal((nw, 2))).astype(dtype)
    off = (0.5 * rng.standard_normal(n)).astype(dtype)
    pairs = op.cell_linked_pairs(np.concatenate((pos, wall)), 2.0 * 1.3 * cfg.dx)
    pairs = pairs[pairs[:, 0] < n]
    T = lambda a: torch.from_numpy(a).to(gpu)
    for kwargs in (dict(nu_field=nu, wall_vel=wv, wall_accel=wa),
                   dict(density_offset=off, wrap_width=1.0)):
        expect = op.rhs(pos, vel, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt, split=True,
                        **kwargs)
        got = rhs(T(pos), T(vel), T(mass), cfg, pairs=T(pairs), wall=T(wall), dt=cfg.dt,
                  split=True, **{k: (T(v) if isinstance(v, np.ndarray) else v)
                                 for k, v in kwargs.items()})
        tr, tf = TOL[np.dtype(dtype)]
        assert rel_err(got[0].cpu(), expect[0]) < tr
        assert rel_err(got[1].cpu(), expect[1], bulk(cfg)) < tr
        assert rel_err(got[2].cpu(), expect[2]) < tf
        assert rel_err(got[3]["reaction"].cpu(), expect[3]["reaction"]) < tf


def test_rhs_pairs_none_and_empty(gpu, default_dtype):
    from tensorsph_b200.droplet_impact import rhs, wall_lattice
    default_dtype(torch.float64)
    cfg = _cfg(dx=0.05, pool_width=0.4, pool_depth=0.15, drop_radius=0.05, drop_center_y=0.25)
    rng = np.random.default_rng(2)
    pos = torch.from_numpy(rng.random((60, 2)) * 0.3).to(gpu)
    vel = torch.zeros_like(pos)
    mass = torch.full((60,), 2.5, dtype=torch.float64, device=gpu)
    wall = wall_lattice(cfg, gpu).double()
    a = rhs(pos, vel, mass, cfg, wall=wall)
    npos = pos.cpu().numpy()
    b = op.rhs(npos, np.zeros_like(npos), mass.cpu().numpy(), cfg, wall=wall.cpu().numpy())
    for x, y in zip(a, b):
        assert rel_err(x.cpu(), y) < 1e-11
    far = torch.tensor([[0.0, 0.0], [10.0, 10.0]], dtype=torch.float64, device=gpu)
    rho, p, acc = rhs(far, torch.zeros_like(far), torch.ones(2, dtype=torch.float64, device=gpu),
                      _cfg(dx=0.1, h_factor=1.0), pairs=torch.empty((0, 2), dtype=torch.long,
                                                                    device=gpu))
    assert torch.equal(acc[:, 0].cpu(), torch.zeros(2, dtype=torch.float64))
    assert torch.allclose(acc[:, 1].cpu(), torch.full((2,), -9.81, dtype=torch.float64))
    with pytest.raises(NotImplementedError):
        rhs(pos, vel, mass, _cfg(surface_tension_coefficient=0.07, csf_scheme="legacy"))


def test_rhs3d_matches_reference(gpu, golden):
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig, rhs_3d
    g = golden("rhs3d")
    for k in range(int(g["count"])):
        cfg = DamBreak3DConfig(dx=0.04, sound_speed=15.0, viscosity=1e-3, dt=1e-4,
                               wall_friction=float(g[f"c{k}_friction"]),
                               density_diffusion=float(g[f"c{k}_diffusion"]))
        t = {name: torch.from_numpy(g[f"c{k}_{name}"]).to(gpu)
             for name in ("pos", "vel", "mass", "wall", "pairs")}
        out = rhs_3d(t["pos"], t["vel"], t["mass"], cfg, pairs=t["pairs"], wall=t["wall"],
                     dt=cfg.dt, return_wall_force=True)
        tr, tf = TOL[g[f"c{k}_pos"].dtype]
        for got, name in zip(out, ("rho", "p", "acc", "reaction")):
            tol = tr if name in ("rho", "p") else tf
            scale = bulk(cfg) if name == "p" else None
            assert rel_err(got.cpu(), g[f"c{k}_{name}"], scale) < tol, (k, name)


def test_rhs_with_csf_matches_reference(golden, gpu):
    """droplet_impact.rhs with CSF surface tension (the fluid pairs of the
    step's list through the 2-D CSF drop-in, droplet_impact.py:1210-1222)
    against the reference's own rhs (tests/golden/rhs_csf.npz, default dtype
    float64): density within 1e-12 of rho0 and the acceleration within 1e-8 of
    the largest surface-tension term, for the default options, "mls" +
    "local_range", and contact angles "rotate" and "young"."""
    import ast
    from dataclasses import replace

    from oracle import csf
    from tensorsph_b200.droplet_impact import Config, rhs
    g = golden("rhs_csf")
    saved = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        for k in range(int(g["count"])):
            o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
            cfg = replace(Config(dx=0.002, pool_width=0.08, pool_depth=0.02, drop_radius=0.01,
                                 drop_center_y=0.035, surface_tension_coefficient=0.0728,
                                 density_diffusion=0.1), **o)
            pos, vel, mass, wall, pairs = (g[f"c{k}_{n}"] for n in ("pos", "vel", "mass", "wall", "pairs"))
            dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
            rho, _, acc = rhs(dev(pos), dev(vel), dev(mass), cfg, pairs=dev(pairs), wall=dev(wall), dt=cfg.dt)
            assert np.abs(rho.cpu().numpy() - g[f"c{k}_rho"]).max() <= 1e-12 * cfg.rho0, k
            n = pos.shape[0]
            fluid = pairs[(pairs[:, 0] < n) & (pairs[:, 1] < n)]
            h = cfg.h_factor * cfg.dx
            a_st, _ = csf.surface_tension_acceleration(
                pos, g[f"c{k}_rho"], mass, h, 0.0728, cfg.rho0, pairs=fluid, curvature_scheme=cfg.csf_curvature,
                delta_normalization=cfg.csf_delta_normalization, wall=wall, contact_angle=cfg.contact_angle,
                contact_angle_model=cfg.contact_angle_model)
            err = np.abs(acc.cpu().numpy() - g[f"c{k}_acc"]).max()
            assert err <= 1e-8 * np.abs(a_st).max(), (k, err / np.abs(a_st).max())
    finally:
        torch.set_default_dtype(saved)


def test_rhs_all_pairs_matches_reference(golden, gpu):
    """rhs_all_pairs against the reference's dense O(N^2) formulation
    (tests/golden/dense.npz, FP64, no walls): density, pressure and
    acceleration within 1e-12 (the "antuono" case keeps the Molteni term, as
    the dense formulation does)."""
    import ast
    from dataclasses import replace

    from tensorsph_b200.droplet_impact import Config, rhs_all_pairs
    g = golden("dense")
    for k in range(int(g["count"])):
        o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
        cfg = replace(Config(dx=0.02, pool_width=0.4, pool_depth=0.15, drop_radius=0.05, drop_center_y=0.25), **o)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        rho, p, acc = rhs_all_pairs(dev(g[f"c{k}_pos"]), dev(g[f"c{k}_vel"]), dev(g[f"c{k}_mass"]), cfg)
        assert np.abs(rho.cpu().numpy() - g[f"c{k}_rho"]).max() <= 1e-12 * cfg.rho0, k
        for name, t in (("p", p), ("acc", acc)):
            ref = g[f"c{k}_{name}"]
            assert np.abs(t.cpu().numpy() - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), (k, name)


def test_regularized_rhs_matches_reference(gpu, golden, default_dtype):
    """The compression density regularisation (rules "free_surface" and
    "internal", normalisations "reference_mean" and "none") and the
    free-surface pressure closure ("interior" with 2 and 3 passes, "all",
    with diffusion, with the boundary-consistent density) against the
    reference's rhs (tests/golden/regularized.npz), FP32 and FP64: two calls
    sharing one state, so the second uses the inverse reference compression
    the first wrote; that scalar and the count are checked too."""
    from tensorsph_b200.droplet_impact import rhs
    from tests.golden.make_golden import REGULARIZED_OPTION_SETS
    g = golden("regularized")
    for k in range(int(g["count"])):
        default_dtype(torch.from_numpy(g[f"c{k}_pos"][:1]).dtype)
        cfg = _cfg(dx=0.05, sound_speed=20.0, viscosity=1e-3, dt=2e-4,
                   **REGULARIZED_OPTION_SETS[int(g[f"c{k}_opts"])])
        t = {name: torch.from_numpy(g[f"c{k}_{name}"]).to(gpu) for name in ("pos", "vel", "mass", "wall", "pairs")}
        tr, tf = TOL[g[f"c{k}_pos"].dtype]
        state = {}
        for call in (0, 1):
            out = rhs(t["pos"], t["vel"], t["mass"], cfg, pairs=t["pairs"], wall=t["wall"], dt=cfg.dt, state=state)
            assert rel_err(out[0].cpu(), g[f"c{k}_rho{call}"]) < tr, (k, call, "rho")
            assert rel_err(out[1].cpu(), g[f"c{k}_p{call}"], bulk(cfg)) < tr, (k, call, "p")
            assert rel_err(out[2].cpu(), g[f"c{k}_acc{call}"]) < tf, (k, call, "acc")
            if f"c{k}_kref{call}" in g:
                kref = state["compression"].inverse_reference_compression
                assert kref == pytest.approx(float(g[f"c{k}_kref{call}"]), rel=tr), (k, call)
                assert state["compression_counted"] == int(g[f"c{k}_counted{call}"]), (k, call)


def test_regularized_rhs_refusals(gpu):
    """The reference's ValueErrors for the compression regularisation."""
    from tensorsph_b200.droplet_impact import rhs
    pos = torch.tensor([[0.0, 0.0], [0.04, 0.0]], dtype=torch.float64, device=gpu)
    for bad in (dict(density_regularization="shepard"),
                dict(density_regularization="compression", density_renormalization=True),
                dict(density_regularization="compression", density_diffusion=0.1),
                dict(density_regularization="compression", compression_regularization_rule="free_stream"),
                dict(density_regularization="compression", compression_normalization="median")):
        with pytest.raises(ValueError):
            rhs(pos, torch.zeros_like(pos), torch.full((2,), 2.5, dtype=torch.float64, device=gpu),
                _cfg(dx=0.05, **bad))


def test_rhs3d_closure_matches_reference(gpu, golden):
    """rhs_3d with the free-surface pressure closure ("interior" with
    diffusion and friction, "all") against the reference's rhs_3d
    (tests/golden/rhs3d_closure.npz), FP32 and FP64."""
    import ast
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig, rhs_3d
    g = golden("rhs3d_closure")
    for k in range(int(g["count"])):
        cfg = DamBreak3DConfig(dx=0.04, sound_speed=15.0, viscosity=1e-3, dt=1e-4,
                               **dict(ast.literal_eval(str(g[f"c{k}_opts"]))))
        t = {name: torch.from_numpy(g[f"c{k}_{name}"]).to(gpu) for name in ("pos", "vel", "mass", "wall", "pairs")}
        out = rhs_3d(t["pos"], t["vel"], t["mass"], cfg, pairs=t["pairs"], wall=t["wall"], dt=cfg.dt,
                     return_wall_force=True)
        tr, tf = TOL[g[f"c{k}_pos"].dtype]
        for got, name in zip(out, ("rho", "p", "acc", "reaction")):
            tol = tr if name in ("rho", "p") else tf
            scale = bulk(cfg) if name == "p" else None
            assert rel_err(got.cpu(), g[f"c{k}_{name}"], scale) < tol, (k, name)


def test_free_stream_rule_raises_after_writing_the_scalar(gpu):
    """rhs passes no indicator, so the rule "free_stream" raises -- after the
    call wrote the new inverse reference compression into the regulariser it
    carries, and without storing the count (compression_regularization.py:
    164-184, droplet_impact.py:1013-1028)."""
    from tensorsph_b200.compression_regularization import CompressionRegularization
    from tensorsph_b200.droplet_impact import rhs
    pos = torch.tensor([[0.0, 0.0], [0.04, 0.0]], dtype=torch.float64, device=gpu)
    reg = CompressionRegularization(rule="free_stream")
    state = {"compression": reg}
    cfg = _cfg(dx=0.05, density_regularization="compression", compression_regularization_rule="free_stream")
    with pytest.raises(ValueError):
        rhs(pos, torch.zeros_like(pos), torch.full((2,), 25.0, dtype=torch.float64, device=gpu), cfg, state=state)
    assert reg.inverse_reference_compression != 1.0 and "compression_counted" not in state
