"""Device checkpoints of the 3-D run (kleefsman_obstacle_3d.py:553-706) and the
obstacle clamp impulse they carry.

* The clamp impulse and the SPH force impulse of the meter rows against the
  FP64 oracle (rhs_3d + Euler + box and obstacle clamps, the clamp taking
  m (v_before - v_after) out, kleefsman_obstacle_3d.py:259-260), on a case
  whose fluid is thrown at the obstacle from all sides: clamp counts equal,
  impulses within 1e-4 of the oracle's largest component.
* Writing checkpoints does not change a run (final positions bit for bit)
  and a completed run removes its file.
* A run stopped after a checkpoint and resumed from it agrees with the run
  that went through: the samples before the checkpoint exactly, the rest to
  round-off (the resumed engine rebuilds its lists at the resume step, so
  its FP32 sums run in another order: positions within 1e-8 m, meters and
  impulses within 1e-6 relative).
* The same for an adaptive-step run, whose checkpoint also carries the
  loop's clock.
"""
import numpy as np
import pytest
import torch

from oracle import pairpass as op
from oracle.neighbors import cell_linked_pairs
from tests.test_gpu_engine import small_case

pytestmark = pytest.mark.gpu

# overlaps the column: the set-up clamp pushes particles to its faces
OBSTACLE = ((0.12, 0.0, 0.04), (0.20, 0.08, 0.16))


def oracle_ledger(cfg, obstacle, x, v, mass, wall, n_ob, steps):
    """Per step (clamps so far, clamp impulse so far, force impulse so far)."""
    x, v = x.copy(), v.copy()
    lo, hi = np.array(obstacle[0]), np.array(obstacle[1])
    box = np.array([cfg.pool_width, cfg.tank_height, cfg.tank_depth])
    tol = 0.25 * cfg.dx
    h = cfg.h_factor * cfg.dx
    clamps, cimp, fimp, out = 0, np.zeros(3), np.zeros(3), []
    for _ in range(steps):
        pairs = cell_linked_pairs(np.concatenate((x, wall)), 2.0 * h)
        _, _, acc, react = op.rhs_3d(x, v, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt,
                                     return_wall_force=True)
        fimp = fimp + react[-n_ob:].sum(axis=0) * cfg.dt
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
            cimp[k] += mass[a] * v[a, k]
            v[a, k] = 0.0
            clamps += 1
        out.append((clamps, cimp.copy(), fimp.copy()))
    return out


def test_clamp_and_force_impulse_match_fp64_oracle(gpu):
    from tensorsph_b200.engine import DamBreak3DEngine
    cfg, _ = small_case()
    x, mass, wall, n_ob = DamBreak3DEngine.build_host_state(cfg, OBSTACLE)
    v0 = torch.zeros_like(x)
    v0[:, 0], v0[:, 1], v0[:, 2] = 8.0, -2.0, 3.0
    steps = 6
    eng = DamBreak3DEngine(cfg, obstacle=OBSTACLE, host_state=(x, mass, wall, n_ob), velocity=v0,
                           diag_ring=64)
    eng.step(steps)
    diag = eng.diagnostics(0, steps).cpu().numpy()
    eng.close()
    ref = oracle_ledger(cfg, OBSTACLE, x.numpy(), v0.numpy(), mass.numpy(), wall.numpy(), n_ob, steps)
    assert ref[-1][0] > 20 and np.count_nonzero(ref[-1][1]) == 3
    cscale = np.abs(ref[-1][1]).max()
    fscale = np.abs(ref[-1][2]).max()
    for k in range(steps):
        clamps, cimp, fimp = ref[k]
        assert int(diag[k, 9]) == clamps, k
        assert np.abs(diag[k, 22:25] - cimp).max() <= 1e-4 * cscale, k
        assert np.abs(diag[k, [14, 20, 21]] - fimp).max() <= 1e-4 * fscale, k


def _cfg(steps):
    from dataclasses import replace
    cfg, _ = small_case()
    return replace(cfg, steps=steps, output_every=4)


def test_checkpoints_leave_the_run_unchanged(gpu, tmp_path):
    from tensorsph_b200.engine import run_case
    cfg = _cfg(12)
    plain = run_case(cfg, obstacle=OBSTACLE)
    path = tmp_path / "state.pt"
    ck = run_case(cfg, obstacle=OBSTACLE, checkpoint_path=path, checkpoint_every=5)
    assert torch.equal(plain.final_positions, ck.final_positions)
    assert plain.times == ck.times and plain.front == ck.front
    assert plain.obstacle_clamps == ck.obstacle_clamps > 0
    assert not path.exists() and not ck.resumed
    assert len(ck.obstacle_impulse) == len(ck.clamp_impulse) == 3


def test_resume_continues_an_interrupted_run(gpu, tmp_path, monkeypatch):
    import pathlib
    from tensorsph_b200.checkpoint import load_checkpoint
    from tensorsph_b200.engine import run_case
    full = run_case(_cfg(20), obstacle=OBSTACLE)
    path = tmp_path / "state.pt"
    # the first attempt stops after 12 steps and keeps its last checkpoint
    # (after the update of step 10), as a process that died would
    with monkeypatch.context() as m:
        m.setattr(pathlib.Path, "unlink", lambda self, missing_ok=False: None)
        run_case(_cfg(12), obstacle=OBSTACLE, checkpoint_path=path, checkpoint_every=5)
    state = load_checkpoint(path, _cfg(20), OBSTACLE)
    assert state["step"] == 10
    assert state["elapsed"] == pytest.approx(11 * _cfg(20).dt, rel=1e-12)
    assert state["times"] == full.times[:3]
    assert state["front"] == full.front[:3]
    assert state["clamps"] <= full.obstacle_clamps
    run = run_case(_cfg(20), obstacle=OBSTACLE, checkpoint_path=path, checkpoint_every=5)
    assert run.resumed and not path.exists()
    assert run.times == full.times
    assert run.front[:3] == full.front[:3]
    np.testing.assert_allclose(run.front, full.front, rtol=1e-9)
    np.testing.assert_allclose(run.kinetic_energy, full.kinetic_energy, rtol=1e-6)
    assert len(run.obstacle_force) == len(full.obstacle_force) == 20
    np.testing.assert_allclose(run.obstacle_force[:11], full.obstacle_force[:11], rtol=1e-12, atol=1e-12)
    f = np.abs(np.array(full.obstacle_force)).max()
    assert np.abs(np.array(run.obstacle_force) - np.array(full.obstacle_force)).max() <= 1e-6 * f
    assert np.abs(np.array(run.obstacle_impulse) - np.array(full.obstacle_impulse)).max() <= \
        1e-6 * np.abs(full.obstacle_impulse).max()
    assert np.abs(np.array(run.clamp_impulse) - np.array(full.clamp_impulse)).max() <= \
        1e-6 * max(np.abs(full.clamp_impulse).max(), 1e-12)
    assert run.obstacle_clamps == full.obstacle_clamps and run.escaped == full.escaped
    assert run.max_density_compression == pytest.approx(full.max_density_compression, rel=1e-6)
    assert run.initial_energy == full.initial_energy
    assert (run.final_positions - full.final_positions).abs().max() < 1e-8


def _adaptive_cfg(steps):
    from dataclasses import replace
    cfg, _ = small_case()
    return replace(cfg, steps=steps, output_every=4, max_courant=0.25, adaptive_dt=True)


def test_adaptive_run_checkpoints_and_resumes(gpu, tmp_path, monkeypatch):
    """adaptive_dt with checkpoints (kleefsman_obstacle_3d.py:598-640): the
    file keeps the loop's clock, the time at the start of the next step and
    the step next_dt chose for it, equal to the uninterrupted run's meter
    rows; checkpointing leaves the run bit for bit unchanged; a run resumed
    from it takes the same number of steps to the same time, its samples
    before the checkpoint exact and the rest to round-off."""
    from tensorsph_b200.checkpoint import load_checkpoint
    from tensorsph_b200.engine import DamBreak3DEngine, _advance_adaptive, run_case
    cfg = _adaptive_cfg(20)
    full = run_case(cfg, obstacle=OBSTACLE)
    eng = DamBreak3DEngine(cfg, obstacle=OBSTACLE, diag_ring=4 * cfg.steps + 1100)
    final = _advance_adaptive(eng, eng.case_id, cfg)
    with torch.cuda.stream(eng.stream):
        diag = eng.diagnostics(0, final + 1).cpu().numpy()
    eng.close()
    assert final == full.steps_taken > cfg.steps and full.dt_min < cfg.dt
    ck = run_case(cfg, obstacle=OBSTACLE, checkpoint_path=tmp_path / "kept.pt", checkpoint_every=5)
    assert torch.equal(ck.final_positions, full.final_positions) and ck.times == full.times
    assert not (tmp_path / "kept.pt").exists()

    path = tmp_path / "state.pt"
    # the first attempt dies right after its checkpoint of step 10 is written
    from tensorsph_b200.checkpoint import CheckpointWriter
    take = CheckpointWriter.take

    class Killed(Exception):
        pass

    def take_then_die(self, step, *a, **kw):
        take(self, step, *a, **kw)
        if step == 10:
            self.wait()
            raise Killed

    with monkeypatch.context() as m:
        m.setattr(CheckpointWriter, "take", take_then_die)
        with pytest.raises(Killed):
            run_case(cfg, obstacle=OBSTACLE, checkpoint_path=path, checkpoint_every=5)
    state = load_checkpoint(path, cfg, OBSTACLE)
    assert state["step"] == 10
    assert state["elapsed"] == diag[11, 25] and state["dt"] == diag[11, 27]
    assert state["times"] == full.times[:3] and state["front"] == full.front[:3]
    run = run_case(cfg, obstacle=OBSTACLE, checkpoint_path=path, checkpoint_every=5)
    assert run.resumed and not path.exists()
    assert run.steps_taken == full.steps_taken
    assert run.simulated_time == pytest.approx(full.simulated_time, rel=1e-12)
    assert run.times[:3] == full.times[:3]
    # the resumed run rebuilds its rows at the checkpoint, so its FP32 sums
    # run in another order: later samples agree to the FP32 round-off of the
    # steps next_dt chooses
    np.testing.assert_allclose(run.times, full.times, rtol=1e-7)
    np.testing.assert_allclose(run.front, full.front, rtol=1e-7)
    np.testing.assert_allclose(run.kinetic_energy, full.kinetic_energy, rtol=1e-6)
    assert len(run.obstacle_force) == len(full.obstacle_force) == final
    np.testing.assert_allclose(run.obstacle_force[:11], full.obstacle_force[:11], rtol=1e-12, atol=1e-12)
    f = np.abs(np.array(full.obstacle_force)).max()
    assert np.abs(np.array(run.obstacle_force) - np.array(full.obstacle_force)).max() <= 1e-6 * f
    assert np.abs(np.array(run.obstacle_impulse) - np.array(full.obstacle_impulse)).max() <= \
        1e-6 * np.abs(full.obstacle_impulse).max()
    assert run.dt_min == pytest.approx(full.dt_min, rel=1e-6) and run.dt_max == full.dt_max
    assert run.max_acoustic_courant == pytest.approx(full.max_acoustic_courant, rel=1e-6)
    assert run.obstacle_clamps == full.obstacle_clamps and run.escaped == full.escaped
    assert run.initial_energy == full.initial_energy
    assert (run.final_positions - full.final_positions).abs().max() < 1e-8
