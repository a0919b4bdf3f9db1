"""The 3-D dam break with the box obstacle (the headline case) on rungs of its
own lattice, engine (FP32 pair arithmetic, FP64 state) against the FP64 oracle
loop (``oracle/dam3d.py``: rhs_3d + Euler + box and obstacle clamps + Lind
shifting, the reference's order).

Rungs: dx = 0.0276 m (29,412 fluid + 49,878 wall particles, 4x the headline
spacing) over several steps, from rest and from the impact on the obstacle;
dx = 0.0138 m (241k fluid, 2x the headline spacing) over one step.

Tolerances are the FP32 bar: density within 1e-5 of rho0 and pressure within
1e-5 of B = rho0 c0^2 / gamma.  The acceleration is compared with its own
yardstick, the largest acceleration of the step: at rest the hydrostatic
balance cancels pressure terms ~1e3 times larger than the net acceleration, so
an FP32 pair sum is ~1e-4 of it away from the FP64 one (the reference's own
FP32 run is 6e-4 away from its FP64 run).  The obstacle force is a sum over
obstacle particles in FP64 of FP32 pair terms; it is compared with its own
magnitude.
"""
import numpy as np
import pytest

from oracle import dam3d

pytestmark = pytest.mark.gpu

RHO_TOL = 1e-5      # |d rho| / rho0
P_TOL = 1e-5        # |d p| / B
ACC_TOL = 2e-4      # |d a| / max |a|
FORCE_TOL = 1e-4    # |d F| / max |F|


def _case(dx):
    from tensorsph_b200.engine import DamBreak3DEngine, obstacle_case
    cfg, obstacle = obstacle_case(dx=dx)
    return cfg, obstacle, DamBreak3DEngine.build_host_state(cfg, obstacle)


def _bulk(cfg):
    return cfg.rho0 * cfg.sound_speed ** 2 / cfg.gamma


def _field_errors(cfg, eng_rho, eng_p, rec):
    return (float(np.abs(eng_rho - rec["rho"]).max()) / cfg.rho0,
            float(np.abs(eng_p - rec["p"]).max()) / _bulk(cfg))


def test_headline_rung_from_rest(gpu):
    """dx = 0.0276: four steps with shifting every step from rest.  The first
    step's density, pressure and velocity, every step's front and peak
    density, and the positions after four steps."""
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle, host = _case(0.0276)
    x, mass, wall, n_ob = host
    steps = 4
    recs, xr, vr = dam3d.run(cfg, obstacle, x.numpy(), mass.numpy(), wall.numpy(), n_ob, steps,
                             shift_every=1)
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=1, host_state=host, diag_ring=64, device=gpu)
    eng.step(1)
    ex, ev, erho, ep = (t.cpu().numpy() for t in eng.state())
    drho, dp = _field_errors(cfg, erho, ep, recs[0])
    assert drho < RHO_TOL and dp < P_TOL, (drho, dp)
    v1 = cfg.dt * recs[0]["acc"]
    dv = float(np.abs(ev - v1).max()) / float(np.abs(v1).max())
    assert dv < ACC_TOL, dv
    eng.step(steps - 1)
    diag = eng.diagnostics(0, steps).cpu().numpy()
    ex, ev, erho, ep = (t.cpu().numpy() for t in eng.state())
    st = eng.status()
    eng.close()
    for k in range(steps):
        assert abs(diag[k, 2] - recs[k]["front"]) < 1e-6 * cfg.dx, k
        assert abs(diag[k, 0] - recs[k]["rho"].max()) < RHO_TOL * cfg.rho0, k
    drho, dp = _field_errors(cfg, erho, ep, recs[-1])
    assert drho < RHO_TOL and dp < P_TOL, (drho, dp)
    assert float(np.abs(ex - xr).max()) < 1e-6 * cfg.dx
    assert st["status"] == 0 and st["steps"] == steps


def test_headline_rung_impact_on_obstacle(gpu):
    """dx = 0.0276: the engine runs from rest until the surge loads the
    obstacle; from that state (positions, velocities, step number) the engine
    and the oracle take three more steps.  Per step: the obstacle force, the
    front and the peak density; after the steps the density and pressure
    fields."""
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle, host = _case(0.0276)
    x, mass, wall, n_ob = host
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=1, host_state=host, diag_ring=8192,
                           device=gpu)
    lead = 0
    f_lead = np.zeros(3)
    while np.abs(f_lead).max() < 1.0 and lead < 8000:   # until the surge loads the obstacle
        eng.step(250)
        lead += 250
        f_lead = eng.diagnostics(lead - 1, 1).cpu().numpy()[0, 3:6]
    eng.step(50)
    lead += 50
    xs, vs, _, _ = (t.cpu() for t in eng.state())
    assert eng.status()["status"] == 0
    eng.close()
    assert np.abs(f_lead).max() >= 1.0, (lead, f_lead)
    steps = 3
    recs, xr, _ = dam3d.run(cfg, obstacle, xs.numpy(), mass.numpy(), wall.numpy(), n_ob, steps,
                            shift_every=1, v0=vs.numpy(), first_step=lead)
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=1, host_state=(xs, mass, wall, n_ob),
                           velocity=vs, first_step=lead, diag_ring=64, device=gpu)
    eng.step(steps)
    diag = eng.diagnostics(lead, steps).cpu().numpy()
    ex, _, erho, ep = (t.cpu().numpy() for t in eng.state())
    eng.close()
    fmax = max(float(np.abs(r["force"]).max()) for r in recs)
    for k in range(steps):
        df = float(np.abs(diag[k, 3:6] - recs[k]["force"]).max()) / fmax
        assert df < FORCE_TOL, (k, df)
        assert abs(diag[k, 2] - recs[k]["front"]) < 1e-6 * cfg.dx, k
        assert abs(diag[k, 0] - recs[k]["rho"].max()) < RHO_TOL * cfg.rho0, k
    drho, dp = _field_errors(cfg, erho, ep, recs[-1])
    assert drho < RHO_TOL and dp < P_TOL, (drho, dp)
    assert float(np.abs(ex - xr).max()) < 1e-5 * cfg.dx


def test_headline_half_rung_one_step(gpu):
    """dx = 0.0138 (241,560 fluid particles): one step from rest without
    shifting; density, pressure and the velocity it produces."""
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle, host = _case(0.0138)
    x, mass, wall, n_ob = host
    recs, _, _ = dam3d.run(cfg, obstacle, x.numpy(), mass.numpy(), wall.numpy(), n_ob, 1)
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, host_state=host, diag_ring=16, device=gpu)
    eng.step(1)
    _, ev, erho, ep = (t.cpu().numpy() for t in eng.state())
    eng.close()
    drho, dp = _field_errors(cfg, erho, ep, recs[0])
    assert drho < RHO_TOL and dp < P_TOL, (drho, dp)
    v1 = cfg.dt * recs[0]["acc"]
    dv = float(np.abs(ev - v1).max()) / float(np.abs(v1).max())
    assert dv < ACC_TOL, dv
