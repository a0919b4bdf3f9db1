"""Host-side logic of the ensemble and the server (no GPU): seeded request
streams, case sizing and the HBM-budget capacities."""
import math

import numpy as np
import pytest


def test_request_stream_is_seeded_poisson():
    from tensorsph_b200.serving import request_stream
    a = request_stream(400, rate=20.0, seed=7)
    b = request_stream(400, rate=20.0, seed=7)
    assert [(r.arrival, r.kind, r.particles) for r in a] == [(r.arrival, r.kind, r.particles) for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 1 / 20.0) < 0.15 / 20.0          # mean inter-arrival 1/rate
    assert min(r.particles for r in a) >= 1000 and max(r.particles for r in a) <= 2_000_000
    logs = np.log([r.particles for r in a])
    assert abs(logs.mean() - 0.5 * (math.log(1e3) + math.log(2e6))) < 0.5   # log-uniform
    assert all(0.1 <= r.sim_time <= 1.0 for r in a)


def test_request_spec_sizes_cases():
    from tensorsph_b200.serving import Request, request_spec
    for kind in ("dam_break_2d", "column_3d"):
        r = Request(0, 0.0, kind, 20000, 0.5, height=1.0)
        spec = request_spec(r)
        assert 0.6 * 20000 < spec.n_fluid < 1.2 * 20000
        assert r.steps == round(0.5 / spec.dt)
        assert spec.cells() > 0


def test_budget_capacities_fit_the_budget():
    from tensorsph_b200.engine import MAX_ROWS, engine_bytes
    from tensorsph_b200.serving import capacities_for_budget
    for budget in (0.25e9, 4e9, 150e9):
        cap = capacities_for_budget(budget)
        assert engine_bytes(**cap) <= budget
        assert cap["max_fluid"] + cap["max_wall"] <= MAX_ROWS
    small = capacities_for_budget(4e9)
    assert engine_bytes(**small) > 0.9 * 4e9


def test_ensemble_draws_follow_the_rules():
    from tensorsph_b200.ensemble import draw_ensemble, droplet_config
    draws = draw_ensemble(256, seed=0)
    assert len(draws) == 256
    for d in draws:
        assert 0.02 <= d.radius <= 0.08 and 2 * d.radius <= d.depth <= 6 * d.radius
        assert 1.0 <= d.speed <= 5.0
        cfg = droplet_config(d)
        assert cfg.dx == pytest.approx(d.radius / 20.0)
        assert cfg.pool_width == pytest.approx(8 * d.radius)
        assert d.speed / cfg.sound_speed <= 0.1 + 1e-12
