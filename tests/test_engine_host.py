"""Host side of the engine's case builders (no GPU): how the droplet case's
CSF options, contact angles and the dam breaks' transport-velocity
correction options become case parameters, and what they refuse."""
import math
from dataclasses import replace

import numpy as np
import pytest
import torch


def _drop(**kw):
    from tensorsph_b200.droplet_impact import Config
    dx = 0.002
    h = 1.3 * dx
    return replace(Config(dx=dx, pool_width=0.08, pool_depth=0.02, drop_radius=0.01, drop_center_y=0.035,
                          sound_speed=20.0, viscosity=1e-6, dt=0.25 * h / 20.0, max_courant=0.25,
                          surface_tension_coefficient=0.0728), **kw)


def test_wall_spacing_matches_oracle():
    from oracle.contact_angle import wall_spacing
    from tensorsph_b200.engine import _wall_spacing
    rng = np.random.default_rng(4)
    for n in (2, 3, 57, 400):
        w = rng.random((n, 2))
        assert _wall_spacing(torch.from_numpy(w)) == wall_spacing(w)
    assert _wall_spacing(torch.zeros((1, 2), dtype=torch.float64)) == 1.0


def test_droplet_csf_options_become_case_parameters():
    from tensorsph_b200.engine import _wall_spacing, droplet_impact_case
    p = droplet_impact_case(_drop()).params
    assert (p.csf_curvature, p.csf_delta_normalization, p.csf_contact_model) == (0, 0, 0)
    p = droplet_impact_case(_drop(csf_curvature="mls", csf_delta_normalization="local_range")).params
    assert (p.csf_curvature, p.csf_delta_normalization) == (1, 1)
    assert droplet_impact_case(_drop(csf_curvature="fit_circle")).params.csf_curvature == 2
    spec = droplet_impact_case(_drop(contact_angle=1.0, contact_angle_reach=1.5))
    assert (spec.params.csf_contact_model, spec.params.csf_contact_angle, spec.params.csf_contact_reach) == (1, 1.0, 1.5)
    assert spec.params.csf_wall_area == 0.0
    spec = droplet_impact_case(_drop(contact_angle=2.0, contact_angle_model="young"))
    assert spec.params.csf_contact_model == 2
    assert spec.params.csf_wall_area == pytest.approx(_wall_spacing(spec.wall) ** 2, rel=0, abs=0)
    assert spec.params.csf_traction_calibration == 0.9611
    assert droplet_impact_case(_drop(contact_angle=2.0, contact_angle_model="brackbill")).params.csf_contact_model == 3
    # without surface tension the options are not carried
    p = droplet_impact_case(_drop(surface_tension_coefficient=0.0, contact_angle=1.0)).params
    assert (p.csf_contact_model, p.surface_tension) == (0, 0.0)


def test_droplet_csf_refusals():
    from tensorsph_b200.engine import droplet_impact_case
    with pytest.raises(NotImplementedError):
        droplet_impact_case(_drop(csf_scheme="legacy"))
    with pytest.raises(NotImplementedError):
        droplet_impact_case(_drop(contact_angle=1.0, contact_angle_reach=2.5))
    with pytest.raises(ValueError):
        droplet_impact_case(_drop(contact_angle=1.0, contact_angle_model="hoffman"))
    with pytest.raises(ValueError):
        droplet_impact_case(_drop(csf_curvature="fit_ellipse"))


def _dam2d(**kw):
    from tensorsph_b200.dam_break import DamBreakConfig
    dx = 0.02
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 0.4)
    return replace(DamBreakConfig(dx=dx, column_width=0.2, column_height=0.4, pool_width=0.6, tank_height=0.6,
                                  sound_speed=c0, dt=0.25 * 1.3 * dx / c0, max_courant=0.25, steps=10), **kw)


def test_dam_break_2d_tvc_options_become_case_parameters():
    from tensorsph_b200.engine import dam_break_2d_case
    h = 1.3 * 0.02
    p = dam_break_2d_case(_dam2d(tvc_every=2)).params
    assert (p.tvc_every, p.tvc_alpha, p.tvc_scope_tol, p.tvc_max_shift, p.tvc_slope, p.tvc_bulk_c) == \
        (2, 0.05, -1.0, -1.0, -1.0, 0.0)
    assert p.tvc_wall_volume == pytest.approx(0.02 ** 2)
    p = dam_break_2d_case(_dam2d(tvc_every=1, tvc_scope="bulk_g", tvc_bulk_g=0.03, tvc_limiter="truncated_linear",
                                 tvc_limiter_slope=7.0, tvc_max_shift=0.1, tvc_alpha=0.2)).params
    assert (p.tvc_scope_tol, p.tvc_slope, p.tvc_alpha) == (0.03, 7.0, 0.2)
    assert p.tvc_max_shift == pytest.approx(0.1 * h)
    p = dam_break_2d_case(_dam2d(tvc_every=1, tvc_scope="bulk", tvc_bulk_c=0.9)).params
    assert (p.tvc_bulk_c, p.tvc_scope_tol) == (0.9, -1.0)
    with pytest.raises(ValueError):
        dam_break_2d_case(_dam2d(tvc_every=1, tvc_scope="bulk", tvc_bulk_c=0.0))
    with pytest.raises(ValueError):
        dam_break_2d_case(_dam2d(tvc_every=1, tvc_limiter="cubic"))
    with pytest.raises(NotImplementedError):
        dam_break_2d_case(_dam2d(tvc_every=1), shift_every=1)


def test_step_limits_match_reference(golden):
    """acoustic_dt_limit, capillary_dt_limit, stable_dt and next_dt against
    values the reference wrote (tests/golden/dt.npz): bit for bit."""
    from tensorsph_b200 import droplet_impact as di
    g = golden("dt")["values"]
    rows = []
    for o in (dict(), dict(viscosity=1e-3), dict(density_diffusion=0.1, surface_tension_coefficient=0.0728),
              dict(dt_growth=0.9, surface_tension_coefficient=0.5, dx=0.001)):
        cfg = di.Config(**o)
        for speed in (0.0, 1.5, 30.0):
            for dt in (cfg.dt, 0.5 * cfg.dt):
                rows.append([di.acoustic_dt_limit(cfg, speed), di.capillary_dt_limit(cfg), di.stable_dt(cfg, speed),
                             di.next_dt(cfg, dt, speed)])
    assert np.array_equal(np.asarray(rows), g)


def test_engine_compression_and_closure_options():
    """The compression regularisation (2-D, droplet_impact.py:982-1028) and
    the free-surface closure (droplet_impact.py:429-492) become case
    parameters; the combinations the rhs refuses raise its ValueErrors, and
    3-D cases ignore the regularisation as rhs_3d does."""
    from tensorsph_b200.engine import dam_break_2d_case, droplet_impact_case
    p = dam_break_2d_case(_dam2d(density_diffusion=0.0, density_regularization="compression")).params
    assert (p.compression, p.compression_rule, p.compression_normalization) == (1, 1, 1)
    p = dam_break_2d_case(_dam2d(density_diffusion=0.0, density_regularization="compression",
                                 compression_regularization_rule="internal",
                                 compression_normalization="none")).params
    assert (p.compression, p.compression_rule, p.compression_normalization) == (1, 0, 0)
    p = dam_break_2d_case(_dam2d(surface_pressure_closure=True, surface_pressure_donors="all",
                                 surface_pressure_threshold=0.98)).params
    assert (p.surface_closure, p.surface_donors, p.surface_threshold) == (1, 1, 0.98)
    p = droplet_impact_case(_drop(surface_pressure_closure=True, surface_pressure_layers=4)).params
    assert (p.surface_closure, p.surface_donors, p.surface_layers) == (1, 0, 4)
    for bad, msg in ((dict(density_diffusion=0.1, density_regularization="compression"), "pick one"),
                     (dict(density_diffusion=0.0, density_regularization="compression",
                           density_renormalization=True), "already-normalised"),
                     (dict(density_diffusion=0.0, density_regularization="compression",
                           compression_regularization_rule="free_stream"), "indicator"),
                     (dict(density_diffusion=0.0, density_regularization="volume"), "unknown")):
        with pytest.raises(ValueError, match=msg):
            dam_break_2d_case(_dam2d(**bad))


def test_dam_break_2d_shift_reference_speed_and_refusals():
    """shift_v_ref (dam_break.py:425-427) becomes the case's fixed shift
    reference speed; surface tension in the dam break is refused."""
    from tensorsph_b200.engine import dam_break_2d_case
    p = dam_break_2d_case(_dam2d(), shift_every=1).params
    assert (p.shift_vref_given, p.shift_vref_floor) == (0, 0.05 * _dam2d().sound_speed)
    p = dam_break_2d_case(_dam2d(shift_v_ref=0.7), shift_every=1).params
    assert (p.shift_vref_given, p.shift_vref) == (1, 0.7)
    with pytest.raises(NotImplementedError):
        dam_break_2d_case(_dam2d(surface_tension_coefficient=0.07))


def test_tuning_cache_roundtrip(tmp_path, monkeypatch):
    """The autotuning cache: a stored best comes back under the same key
    only (workload, particle count to 3 significant digits, candidates, GPU)."""
    from tensorsph_b200 import tuning
    monkeypatch.setenv("TSPH_TUNING_CACHE", str(tmp_path / "t.json"))
    k1 = tuning.tuning_key("dam_break_3d", dim=3, particles=1968048, h_over_dx=1.3,
                           candidates={"skins": (0.1, 0.15)}, gpu="NVIDIA B200")
    k2 = tuning.tuning_key("dam_break_3d", dim=3, particles=1968400, h_over_dx=1.3,
                           candidates={"skins": (0.1, 0.15)}, gpu="NVIDIA B200")
    k3 = tuning.tuning_key("dam_break_3d", dim=3, particles=1968048, h_over_dx=1.3,
                           candidates={"skins": (0.1, 0.15)}, gpu="NVIDIA H100")
    assert k1 == k2 and k1 != k3
    assert tuning.lookup(k1) is None
    tuning.store(k1, {"skin_factor": 0.15, "block": 128, "batch": 8})
    assert tuning.lookup(k2) == {"skin_factor": 0.15, "block": 128, "batch": 8}
    assert tuning.lookup(k3) is None


def test_tuner_prefers_the_wider_skin_among_equal_trials():
    """Trials from rest cannot see the rebuilds a wider skin saves later, so a
    near-tie goes to the wider skin; a clear win by a narrower one stands."""
    from tensorsph_b200.engine import pick_trial
    trials = [{"skin_factor": 0.10, "batch": 4, "ms_per_step": 1.870},
              {"skin_factor": 0.15, "batch": 8, "ms_per_step": 1.880},
              {"skin_factor": 0.15, "batch": 4, "ms_per_step": 1.884},
              {"skin_factor": 0.25, "batch": 8, "ms_per_step": 2.050}]
    assert pick_trial(trials) == trials[1]
    trials[0]["ms_per_step"] = 1.80
    assert pick_trial(trials) == trials[0]


def test_fixed_point_row_test_lists_every_pair_within_the_cutoff():
    """The row builder's criterion, restated: positions rounded to units of a
    power-of-two q with 2^31 q >= the extent, squared integer distance against
    ceil((cutoff / q + 2)^2).  It lists every pair within the cutoff (FP64) and
    nothing beyond the cutoff plus (2 + sqrt(3)) q (seeded cloud with pairs
    placed on the cutoff)."""
    import math
    import numpy as np
    rng = np.random.default_rng(7)
    extent, rc = 3.3, 0.0193
    k = -60
    while math.ldexp(1.0, k + 31) < extent:
        k += 1
    q = math.ldexp(1.0, k)
    a = rng.uniform(0.0, extent, (4000, 3))
    d = rng.normal(size=(4000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    b = a + d * (rc + rng.uniform(-3 * q, 3 * q, (4000, 1)))   # pairs straddling the cutoff
    r = np.linalg.norm(a - b, axis=1)
    ia = np.rint(a / q).astype(np.int64)
    ib = np.rint(b / q).astype(np.int64)
    d2 = ((ia - ib) ** 2).sum(axis=1)
    lim = math.ceil((rc / q + 2.0) ** 2)
    listed = d2 <= lim
    assert listed[r <= rc].all()
    assert (r[listed] <= rc + (2.0 + math.sqrt(3.0)) * q * (1 + 1e-9)).all()
