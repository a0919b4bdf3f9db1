"""The device engine against the FP64 oracle: one step and a short run.

The engine computes pair arithmetic in FP32 (FP64 separations, compensated
sums) and integrates in FP64; the oracle runs the reference algorithm
(``rhs_3d`` + semi-implicit Euler + box and obstacle clamps) in FP64 with a
fresh pair list every step.  Tolerances: density |d rho| / rho0 < 1e-5,
pressure |d p| / B < 1e-5, velocity after one step |d v| / max|v| < 2e-4
(the hydrostatic balance cancels pressure terms ~1e3 times larger than the
net acceleration), obstacle force within 1e-4 of its FP64 value.
"""
import math

import numpy as np
import pytest
import torch

from oracle import pairpass as op
from oracle.neighbors import cell_linked_pairs

pytestmark = pytest.mark.gpu


def small_case(shift_every=0):
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 0.24)
    dx = 0.02
    h = 1.3 * dx
    cfg = DamBreak3DConfig(dx=dx, pool_width=0.5, tank_depth=0.2, tank_height=0.4,
                           column_width=0.2, column_depth=0.2, column_height=0.24,
                           sound_speed=c0, viscosity=1e-3, dt=0.25 * h / c0,
                           density_diffusion=0.1, wall_friction=0.3, steps=12, output_every=4)
    obstacle = ((0.22, 0.0, 0.04), (0.30, 0.08, 0.16))
    return cfg, obstacle


def oracle_steps(cfg, obstacle, x, mass, wall, n_ob, steps):
    """FP64 oracle trajectory; returns per-step (rho, p, force) and the final state."""
    x = x.copy()
    v = np.zeros_like(x)
    out = []
    lo, hi = np.array(obstacle[0]), np.array(obstacle[1])
    box = np.array([cfg.pool_width, cfg.tank_height, cfg.tank_depth])
    tol = 0.25 * cfg.dx
    for _ in range(steps):
        h = cfg.h_factor * cfg.dx
        pairs = cell_linked_pairs(np.concatenate((x, wall)), 2.0 * h)
        rho, p, acc, react = op.rhs_3d(x, v, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt,
                                       return_wall_force=True)
        out.append((rho, p, react[-n_ob:].sum(axis=0), acc))
        v = v + cfg.dt * acc
        x = x + cfg.dt * v
        out_mask = (x < -tol) | (x > box + tol)
        x = np.clip(x, 0.0, box)
        v[out_mask] = 0.0
        inside = np.all((x > lo) & (x < hi), axis=1)
        for a in np.nonzero(inside)[0]:
            cand = [x[a, 0] - lo[0], hi[0] - x[a, 0], x[a, 1] - lo[1], hi[1] - x[a, 1],
                    x[a, 2] - lo[2], hi[2] - x[a, 2]]
            f = int(np.argmin(cand))
            k = f // 2
            x[a, k] = hi[k] + 0.01 * cfg.dx if f % 2 else lo[k] - 0.01 * cfg.dx
            v[a, k] = 0.0
    return out, x, v


@pytest.mark.parametrize("opts", [dict(), dict(surface_pressure_closure=True, surface_pressure_layers=3)])
def test_engine_matches_fp64_oracle(opts, gpu):
    """The 3-D obstacle case against the FP64 oracle (rhs_3d, Euler, box and
    obstacle clamps), with and without rhs_3d's free-surface pressure closure
    (dam_break_3d.py:339-342)."""
    from dataclasses import replace
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle = small_case()
    cfg = replace(cfg, **opts)
    x, mass, wall, n_ob = DamBreak3DEngine.build_host_state(cfg, obstacle)
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, host_state=(x, mass, wall, n_ob), diag_ring=64)
    steps = 8
    ref, xr, vr = oracle_steps(cfg, obstacle, x.numpy(), mass.numpy(), wall.numpy(), n_ob, steps)
    eng.step(1)
    ex, ev, erho, ep = [t.cpu().numpy() for t in eng.state()]
    bulk = cfg.rho0 * cfg.sound_speed ** 2 / cfg.gamma
    rho0, p0, f0, acc0 = ref[0]
    assert np.abs(erho - rho0).max() / cfg.rho0 < 1e-5
    assert np.abs(ep - p0).max() / bulk < 1e-5
    v1 = cfg.dt * acc0
    assert np.abs(ev - v1).max() / np.abs(v1).max() < 2e-4
    eng.step(steps - 1)
    diag = eng.diagnostics(0, steps).cpu().numpy()
    for k in range(steps):
        fk = ref[k][2]
        assert np.abs(diag[k, 3:6] - fk).max() <= 1e-4 * max(np.abs(fk).max(), 1e-12) + 1e-9, k
        assert diag[k, 0] == pytest.approx(ref[k][0].max(), rel=2e-6)
    ex, ev, _, _ = [t.cpu().numpy() for t in eng.state()]
    assert np.abs(ex - xr).max() < 1e-6 * cfg.dx * steps
    assert np.abs(ev - vr).max() / max(np.abs(vr).max(), 1e-12) < 5e-4
    st = eng.status()
    assert st["steps"] == steps and st["rebuilds"] >= 1 and st["status"] == 0
    eng.close()


def test_engine_shift_matches_fp64_oracle(gpu):
    """Lind shifting in the engine against the oracle.  Two steps (the engine
    shifts from its second step on, with the maximum speed at the start of
    that step as v_ref) with a zero skin, so that both list passes of every
    step rebuild and permute rows; the FP64 side is rhs_3d + Euler + clamps
    and then shift_positions.  The lattice is jittered by +-0.1 dx so that
    the concentration gradient is nonzero in the bulk.

    The shift of this case is small (the reference normalises the 3-D
    concentration with the 2-D kernel constant, so C ~ 0.04 and the shift
    ~4e-6 dx), so it is compared as a displacement: the engine run with
    shifting minus the same run without, against the oracle's shift vector,
    to 1e-5 of its largest component (measured 4e-7).  Positions without
    the shift agree with the oracle to 1e-6 dx (measured 3e-8 dx)."""
    from dataclasses import replace
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle = small_case()
    cfg = replace(cfg, pair_skin_factor=0.0)
    x, mass, wall, n_ob = DamBreak3DEngine.build_host_state(cfg, obstacle)
    rng = np.random.default_rng(7)
    x = (x + torch.from_numpy(rng.uniform(-0.1, 0.1, tuple(x.shape)) * cfg.dx)).clamp(min=0.0)
    runs, first_rho = {}, {}
    for every in (0, 1):
        eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=every,
                               host_state=(x, mass, wall, n_ob), diag_ring=64)
        eng.step(1)
        # read back after the second list pass of step 0 rebuilt and
        # permuted the rows: the density stays with its particle
        first_rho[every] = eng.state()[2].cpu().numpy()
        eng.step(1)
        runs[every] = eng.state()[0].cpu().numpy()
        st = eng.status()
        if every:
            eng.step(1)   # the meter row of step 2 reports the c_ref of step 1's shift
            c_ref = float(eng.diagnostics(2, 1).cpu()[0, 15])
        eng.close()
        assert st["status"] == 0 and st["rebuilds"] >= 2 + every
    xn, mn, wn = x.numpy(), mass.numpy(), wall.numpy()
    _, _, v1 = oracle_steps(cfg, obstacle, xn, mn, wn, n_ob, 1)
    ref, x2, _ = oracle_steps(cfg, obstacle, xn, mn, wn, n_ob, 2)
    h = cfg.h_factor * cfg.dx
    vref = max(float(np.linalg.norm(v1, axis=1).max()), 0.05 * cfg.sound_speed)
    _, info = op.shift_positions(x2, mn / ref[1][0], h, dt=cfg.dt, v_ref=vref, strength=1.0,
                                 limit=0.25, free_surface=0.95)
    shift = info["shift"]
    for every in (0, 1):
        assert np.abs(first_rho[every] - ref[0][0]).max() / cfg.rho0 < 1e-5
    # the device radix select of the 95th percentile against np.quantile
    assert c_ref == pytest.approx(info["c_reference"], rel=1e-5)
    assert np.abs(shift).max() > 1e-6 * cfg.dx
    assert np.abs(runs[0] - x2).max() < 1e-6 * cfg.dx
    err = np.abs((runs[1] - runs[0]) - shift).max()
    assert err < 1e-5 * np.abs(shift).max(), err / np.abs(shift).max()


@pytest.mark.parametrize("opts", [dict(), dict(tvc_alpha=0.2, tvc_scope_tol=0.05, tvc_max_shift=1e-4)])
def test_engine_tvc_matches_fp64_oracle(opts, gpu):
    """Transport-velocity correction in the engine (dam_break_3d.py:675-704)
    against the oracle: two steps (the correction runs after the update of
    step 1), a zero skin so that the rows are the step's 2h pairs at its
    start, as the reference's cache hands them over, from a lattice jittered
    by +-0.1 dx.  The displacement (run with the correction minus run
    without) matches the oracle's shift to 1e-5 of its largest component
    (1e-4 with the clip: it scales bulk particles, whose g is a strongly
    cancelling FP32 sum with ~1e-5 relative error, up to the full clip
    length), and the logged max / mean shift and clipped fraction match."""
    from dataclasses import replace
    from oracle import tvc as otv
    from tensorsph_b200.dam_break_3d import mass_3d
    from tensorsph_b200.engine import DamBreak3DEngine, run_case
    cfg, _ = small_case()
    cfg = replace(cfg, pair_skin_factor=0.0, steps=2, output_every=1)
    x, mass, wall, n_ob = DamBreak3DEngine.build_host_state(cfg, None)
    rng = np.random.default_rng(9)
    x = (x + torch.from_numpy(rng.uniform(-0.1, 0.1, tuple(x.shape)) * cfg.dx)).clamp(min=0.0)
    runs = {}
    for every in (0, 1):
        c = replace(cfg, tvc_every=every, **opts)
        eng = DamBreak3DEngine(c, host_state=(x, mass, wall, n_ob), diag_ring=64)
        eng.step(2)
        runs[every] = eng.state()[0].cpu().numpy()
        diag = eng.diagnostics(1, 1).cpu().numpy()[0]
        assert eng.status()["status"] == 0
        eng.close()
    xn, mn, wn = x.numpy(), mass.numpy(), wall.numpy()
    ref, x2, _ = oracle_steps(cfg, ((9, 9, 9), (9, 9, 9)), xn, mn, wn, 0, 2)
    _, x1, _ = oracle_steps(cfg, ((9, 9, 9), (9, 9, 9)), xn, mn, wn, 0, 1)
    h = cfg.h_factor * cfg.dx
    pairs = cell_linked_pairs(np.concatenate((x1, wn)), 2.0 * h)
    wvol = mass_3d(cfg.dx, cfg.h_factor, cfg.rho0, cfg.density_calibration) / cfg.rho0
    vol = np.concatenate((mn / ref[1][0], np.full(wn.shape[0], wvol)))
    c = replace(cfg, tvc_every=1, **opts)
    res = otv.transport_velocity_correction(
        np.concatenate((x2, wn)), vol, h, pairs, wall_count=wn.shape[0],
        alpha=0.05 if c.tvc_alpha is None else c.tvc_alpha, h_ref=h, scope_tol=c.tvc_scope_tol,
        max_shift=None if c.tvc_max_shift is None else c.tvc_max_shift * h)
    shift = res["shift"]
    assert np.abs(shift).max() > 1e-4 * cfg.dx
    err = np.abs((runs[1] - runs[0]) - shift).max()
    tol = 1e-4 if c.tvc_max_shift is not None else 1e-5
    assert err < tol * np.abs(shift).max(), err / np.abs(shift).max()
    norm = np.linalg.norm(shift, axis=1)
    assert diag[16] == pytest.approx(norm.max(), rel=1e-5)
    assert diag[17] == pytest.approx(norm.sum(), rel=1e-5)
    assert diag[19] / mn.size == pytest.approx(res["clipped"], abs=1.5 / mn.size)
    log = run_case(replace(cfg, tvc_every=1, steps=3, **opts)).tvc_log
    assert [e["step"] for e in log] == [1, 2]


def test_engine_shift_runs_and_moves_particles(gpu):
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle = small_case()
    a = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=1, diag_ring=64)
    b = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=0, diag_ring=64)
    a.step(6)
    b.step(6)
    xa = a.state()[0]
    xb = b.state()[0]
    d = (xa - xb).norm(dim=1)
    assert torch.isfinite(xa).all()
    assert float(d.max()) > 0.0
    assert float(d.max()) < 6 * 0.25 * cfg.h_factor * cfg.dx
    diag = a.diagnostics(0, 6).cpu()
    assert float(diag[5, 15]) > 0.0  # c_ref from the device radix select
    a.close()
    b.close()


def test_engine_graph_and_eager_agree(gpu):
    """The step graph (its list rebuild in a conditional node that only runs
    when a case is due) and kernel-by-kernel launches give the same run, with
    a zero skin so that both list passes rebuild on every step."""
    from dataclasses import replace
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, obstacle = small_case()
    cfg = replace(cfg, pair_skin_factor=0.0)   # any motion rebuilds: both passes of every step
    a = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=1, diag_ring=64)
    b = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=1, diag_ring=64)
    a.step(12, graph=True)
    b.step(12, graph=False)
    for u, w in zip(a.state(), b.state()):
        assert torch.equal(u, w)
    sa, sb = a.status(), b.status()
    assert sa["rebuilds"] == sb["rebuilds"] > 4
    every, per_rebuild = a.graph_kernels()
    assert every > 10 and per_rebuild > 5
    a.close()
    b.close()


def test_run_case_record(gpu):
    from tensorsph_b200.engine import run_case
    cfg, obstacle = small_case()
    run = run_case(cfg, obstacle=obstacle)
    assert run.steps_taken == cfg.steps
    assert len(run.times) == len(run.front) == 4      # steps 0, 4, 8 and the final 12
    assert run.front[0] == pytest.approx(0.19, abs=1e-9)
    assert run.escaped == 0
    assert len(run.obstacle_force) == cfg.steps


def test_run_case_snapshots(gpu):
    """snapshot_times as the reference loop takes them: each target at the
    first sample point (every output_every steps and the last) whose time
    reaches it, several targets may share one, targets past the end are not
    taken; the copies (made on a side stream while the loop goes on) equal
    the state of a plain run stopped at that step."""
    from tensorsph_b200.engine import DamBreak3DEngine, run_case
    cfg, obstacle = small_case()      # 12 steps, samples at 0, 4, 8, 12
    dt = cfg.dt
    run = run_case(cfg, obstacle=obstacle, snapshot_times=[0.0, 0.5 * dt, 4 * dt, 9.5 * dt, 100.0])
    assert [round(t / dt, 9) for t, _, _ in run.snapshots] == [0, 4, 4, 12]
    assert torch.equal(run.snapshots[-1][1], run.final_positions)
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, diag_ring=64)
    eng.step(4)
    x, v, _, _ = (t.cpu() for t in eng.state())
    eng.close()
    for _, sx, sv in run.snapshots[1:3]:
        assert torch.equal(sx, x) and torch.equal(sv, v)
    assert torch.equal(run.snapshots[0][1], run_case(cfg, obstacle=obstacle,
                                                     snapshot_times=[0.0]).snapshots[0][1])


def test_run_case_follows_reference_run(golden, gpu):
    """The small 3-D dam break (Molteni diffusion, wall friction, 40 steps) on
    the device against the reference's own FP64 ``dam_break_3d.run_case``."""
    from tensorsph_b200.engine import run_case
    g = golden("dam3d_run")
    cfg, _ = small_case()
    from dataclasses import replace
    cfg = replace(cfg, steps=40, output_every=10)
    saved = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        run = run_case(cfg)
    finally:
        torch.set_default_dtype(saved)
    from tests.trajectory import assert_follows
    assert_follows(run, g, front_tol=1e-7)
    assert run.max_speed == pytest.approx(float(g["max_speed"]), rel=1e-4)
    from tensorsph_b200.engine import DamBreak3DEngine
    x0 = DamBreak3DEngine.build_host_state(cfg)[0].numpy()
    moved = np.abs(g["final_positions"] - x0).max()
    dxmax = np.abs(run.final_positions.numpy() - g["final_positions"]).max()
    assert dxmax < 1e-4 * moved, (dxmax, moved)


def test_adaptive_3d_run_with_obstacle(gpu):
    """adaptive_dt in the 3-D loop (dam_break_3d.py:617-711) with the
    obstacle: at max_courant 0.25 the step shrinks to dt_safety of the
    acoustic limit at once, so the run takes more steps than the fixed one
    to reach steps * dt; each step against next_dt, the obstacle impulse as
    the sum of force times step, and the fixed-step record unchanged when the
    limit never binds."""
    from dataclasses import replace
    from tensorsph_b200.engine import DamBreak3DEngine, _advance_adaptive, run_case
    from tests.test_gpu_batch import assert_adaptive_rows
    cfg, obstacle = small_case()
    cfg = replace(cfg, steps=30, output_every=10, max_courant=0.25, adaptive_dt=True)
    saved = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        run = run_case(cfg, obstacle=obstacle)
        eng = DamBreak3DEngine(cfg, obstacle=obstacle, max_neighbors=160, diag_ring=4 * cfg.steps + 1100)
        final = _advance_adaptive(eng, eng.case_id, cfg)
        with torch.cuda.stream(eng.stream):
            diag = eng.diagnostics(0, final + 1).cpu()
        eng.close()
        # max_courant 0.6: the target step stays above dt, so only the last
        # step could be clipped and the record is the fixed-step one
        loose = replace(cfg, max_courant=0.6)
        a, f = run_case(loose, obstacle=obstacle), run_case(replace(loose, adaptive_dt=False), obstacle=obstacle)
    finally:
        torch.set_default_dtype(saved)
    assert final == run.steps_taken > cfg.steps
    assert_adaptive_rows(cfg, diag, final)
    d = diag.numpy()
    assert run.dt_max == cfg.dt and run.dt_min == pytest.approx(0.9 * cfg.dt, rel=0.05)
    assert run.simulated_time == pytest.approx(cfg.steps * cfg.dt, rel=1e-12)
    assert run.times == [float(d[k, 25]) for k in range(final + 1) if k % 10 == 0 or k == final]
    impulse = sum(float(d[k, 3]) * float(d[k, 26]) for k in range(final))
    assert run.obstacle_impulse[0] == pytest.approx(impulse, rel=1e-12, abs=1e-15)
    assert len(run.obstacle_force) == final
    assert a.steps_taken == f.steps_taken == cfg.steps and a.dt_min == a.dt_max == cfg.dt
    assert np.allclose(a.times, f.times, rtol=1e-12, atol=0)
    for key in ("front", "kinetic_energy", "potential_energy"):
        assert np.allclose(getattr(a, key), getattr(f, key), rtol=1e-9, atol=1e-12), key
    # the final step's size is clipped to the target time (about 0), so its
    # speed, counted in the fixed run's Courant peak, adds nothing here
    assert a.max_speed == pytest.approx(f.max_speed, rel=1e-9)
    assert a.max_acoustic_courant <= f.max_acoustic_courant
