"""CSF surface tension in the device engine against the FP64 oracle
(oracle/csf.py, pinned to the reference's own outputs).

The engine runs the CSF passes in FP64 on the FP64 positions (the operator
differentiates the colour twice and divides by |grad c|: the reference's own
FP32 run is 0.4-1 % away from its FP64 run on these drops).  The
surface-tension acceleration is isolated as the difference of one step with
and without sigma and compared with the oracle's a = -sigma kappa delta_s n /
rho: within 1e-5 of max |a| (the density it divides by comes from the FP32
pair pass).
"""
import numpy as np
import pytest
import torch

from oracle import csf
from oracle import pairpass as op
from oracle.neighbors import cell_linked_pairs

pytestmark = pytest.mark.gpu


def drop_config(sigma):
    from tensorsph_b200.droplet_impact import Config
    dx = 0.002
    h = 1.3 * dx
    c0 = 20.0
    return Config(dx=dx, pool_width=0.08, pool_depth=0.02, drop_radius=0.01, drop_center_y=0.035,
                  sound_speed=c0, viscosity=1e-6, dt=0.25 * h / c0, max_courant=0.25,
                  surface_tension_coefficient=sigma)


@pytest.mark.parametrize("curvature,normalization", [("fit_quadratic", "legacy"), ("mls", "legacy"),
                                                     ("mls", "local_range"), ("fit_quadratic", "local_range"),
                                                     ("fit_circle", "legacy")])
def test_engine_csf_matches_oracle(curvature, normalization, gpu):
    """The droplet case's CSF options (csf_curvature, csf_delta_normalization).
    With "mls" the reference hands the CSF the step's cached fluid list, so the
    oracle gets the fluid pairs within 2h + skin of the first build (what
    "local_range" reads); the fits use the 4h list the reference builds."""
    from dataclasses import replace

    from tensorsph_b200.engine import BatchEngine, capacity_for, droplet_impact_case
    got = {}
    for sigma in (0.0728, 0.0):
        cfg = replace(drop_config(sigma), csf_curvature=curvature, csf_delta_normalization=normalization)
        spec = droplet_impact_case(cfg)
        eng = BatchEngine(**capacity_for([spec], max_neighbors=64, diag_ring=8))
        cid = eng.add(spec)
        eng.step(1)
        got[sigma] = eng.read(cid)[1].cpu().numpy()
        eng.close()
    cfg = replace(drop_config(0.0728), csf_curvature=curvature, csf_delta_normalization=normalization)
    x, m, w = spec.x.numpy(), spec.mass.numpy(), spec.wall.numpy()
    h = cfg.h_factor * cfg.dx
    pairs = cell_linked_pairs(np.concatenate((x, w)), 2.0 * h)
    rho, _, _ = op.rhs(x, np.zeros_like(x), m, cfg, pairs=pairs, wall=w, dt=cfg.dt)
    listed = cell_linked_pairs(x, (2.0 + cfg.pair_skin_factor) * h) if curvature == "mls" else None
    a_ref, st = csf.surface_tension_acceleration(x, rho, m, h, 0.0728, cfg.rho0, pairs=listed,
                                                 curvature_scheme=curvature, delta_normalization=normalization)
    a_dev = (got[0.0728] - got[0.0]) / cfg.dt
    scale = np.abs(a_ref).max()
    err = np.abs(a_dev - a_ref).max(axis=1) / scale
    assert scale > 0.1
    assert err.max() < 1e-5, (err.max(), int(err.argmax()), int((err > 1e-6).sum()))


def test_csf_batch_equals_alone(gpu):
    from tensorsph_b200 import ensemble as en
    from tensorsph_b200.engine import BatchEngine, capacity_for
    specs = en.ensemble_specs(en.draw_ensemble(4, seed=5))
    eng = BatchEngine(**capacity_for(specs, max_neighbors=64, diag_ring=8))
    ids = [eng.add(s) for s in specs]
    eng.step(5)
    eng.remove(ids[1])
    eng.step(3)
    got = {i: [t.cpu() for t in eng.read(i)] for i in (ids[0], ids[2], ids[3])}
    eng.close()
    for i, spec in ((ids[0], specs[0]), (ids[2], specs[2]), (ids[3], specs[3])):
        e2 = BatchEngine(**capacity_for([spec], max_neighbors=64, diag_ring=8))
        j = e2.add(spec)
        e2.step(8)
        ref = [t.cpu() for t in e2.read(j)]
        e2.close()
        for u, v in zip(got[i], ref):
            assert torch.equal(u, v)


@pytest.mark.parametrize("model,theta", [("rotate", np.pi / 3), ("young", 2 * np.pi / 3), ("brackbill", np.pi / 3)])
def test_engine_csf_contact_angle_matches_oracle(model, theta, gpu):
    """Contact angles in the engine's CSF (the droplet case's contact_angle,
    contact_angle_model) against the oracle on a drop above a walled pool
    (positions jittered by 0.02 dx so that no fluid particle is equidistant
    from two wall particles): the surface-tension acceleration within 1e-5 of
    max |a|, and for the tractions the traction alone (with the contact angle
    minus without) within four FP32 steps of the total acceleration the
    engine records (plus 1e-5 of the traction's largest value)."""
    from dataclasses import replace

    from tensorsph_b200.engine import BatchEngine, capacity_for, droplet_impact_case
    rng = np.random.default_rng(21)
    base = droplet_impact_case(drop_config(0.0728))
    x = base.x + torch.from_numpy(rng.uniform(-0.02, 0.02, tuple(base.x.shape)) * 0.002)

    def run(cfg):
        spec = droplet_impact_case(cfg)
        spec.x = x.clone()
        eng = BatchEngine(**capacity_for([spec], max_neighbors=64, diag_ring=8))
        cid = eng.add(spec)
        eng.step(1)
        v = eng.read(cid)[1].cpu().numpy()
        eng.close()
        return v

    with_ca = replace(drop_config(0.0728), contact_angle=float(theta), contact_angle_model=model)
    got = run(with_ca)
    bare = run(drop_config(0.0728))
    zero = run(drop_config(0.0))
    cfg = with_ca
    xn, m, w = x.numpy(), base.mass.numpy(), base.wall.numpy()
    h = cfg.h_factor * cfg.dx
    pairs = cell_linked_pairs(np.concatenate((xn, w)), 2.0 * h)
    rho, _, _ = op.rhs(xn, np.zeros_like(xn), m, cfg, pairs=pairs, wall=w, dt=cfg.dt)
    a_ref, _ = csf.surface_tension_acceleration(xn, rho, m, h, 0.0728, cfg.rho0, wall=w, contact_angle=float(theta),
                                                contact_angle_model=model)
    a_bare, _ = csf.surface_tension_acceleration(xn, rho, m, h, 0.0728, cfg.rho0)
    a_dev = (got - zero) / cfg.dt
    scale = np.abs(a_ref).max()
    assert np.abs(a_ref - a_bare).max() > 1e-4 * scale          # the contact angle acts
    err = np.abs(a_dev - a_ref).max() / scale
    assert err < 1e-5, err
    if model != "rotate":
        # the engine stores the step's total acceleration in FP32 (~10 m/s^2
        # of gravity and pressure); the traction (~1e-3 of the CSF term) is
        # resolved to a few FP32 steps of that total
        t_ref = a_ref - a_bare
        t_dev = (got - bare) / cfg.dt
        ulp = float(np.spacing(np.float32(np.abs(got / cfg.dt).max())))
        terr = np.abs(t_dev - t_ref).max()
        assert terr <= 4 * ulp + 1e-5 * np.abs(t_ref).max(), (terr, ulp, np.abs(t_ref).max())
