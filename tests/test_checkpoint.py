"""Checkpoint format of the 3-D obstacle case (kleefsman_obstacle_3d.py:477-546)
against a file the reference wrote (tests/golden/checkpoint.npz): the same
version, fingerprint fields, keys and values; refusal of another
configuration or version; the atomic replace.  Host only."""
import json
import types

import numpy as np
import pytest
import torch

from tensorsph_b200 import checkpoint as ck


def _cfg(fingerprint: dict):
    return types.SimpleNamespace(**fingerprint)


def _reference_file(golden, tmp_path):
    g = golden("checkpoint")
    path = tmp_path / "state.pt"
    path.write_bytes(g["raw"].tobytes())
    return g, path


def test_fingerprint_fields_and_version_match_reference(golden):
    g = golden("checkpoint")
    assert int(g["version"]) == ck.CHECKPOINT_VERSION
    assert json.loads(str(g["fields"])) == list(ck.CHECKPOINT_FINGERPRINT_FIELDS)
    fp = json.loads(str(g["fingerprint"]))
    assert ck.checkpoint_fingerprint(_cfg(fp)) == fp


def test_reference_checkpoint_loads_and_round_trips(golden, tmp_path):
    g, path = _reference_file(golden, tmp_path)
    fp = json.loads(str(g["fingerprint"]))
    ref = ck.load_checkpoint(path, _cfg(fp))
    args = json.loads(str(g["args"]))
    series = json.loads(str(g["series"]))
    assert torch.equal(ref["positions"], torch.from_numpy(g["pos"]))
    assert torch.equal(ref["velocity"], torch.from_numpy(g["vel"]))
    # the same inputs through this writer give the same payload
    run = types.SimpleNamespace(**series)
    ours_path = tmp_path / "ours.pt"
    ck.save_checkpoint(ours_path, _cfg(fp), positions=torch.from_numpy(g["pos"]),
                       velocity=torch.from_numpy(g["vel"]), run=run, **args)
    ours = torch.load(ours_path, map_location="cpu", weights_only=False)
    assert set(ours) == set(ref)
    for k, v in ref.items():
        if isinstance(v, torch.Tensor):
            assert torch.equal(ours[k], v) and ours[k].dtype == v.dtype, k
        else:
            assert ours[k] == v and type(ours[k]) is type(v), k
    assert not (tmp_path / "ours.pt.tmp").exists()


def test_load_refuses_other_configuration_and_version(golden, tmp_path):
    g, path = _reference_file(golden, tmp_path)
    fp = json.loads(str(g["fingerprint"]))
    other = dict(fp, dx=fp["dx"] * 2)
    with pytest.raises(ValueError, match="different configuration: dx"):
        ck.load_checkpoint(path, _cfg(other))
    payload = torch.load(path, map_location="cpu", weights_only=False)
    payload["version"] = 2
    torch.save(payload, tmp_path / "v2.pt")
    with pytest.raises(ValueError, match="version 2 != 3"):
        ck.load_checkpoint(tmp_path / "v2.pt", _cfg(fp))


def test_t_end_and_steps_are_not_in_the_fingerprint():
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig
    a = ck.checkpoint_fingerprint(DamBreak3DConfig(steps=10))
    b = ck.checkpoint_fingerprint(DamBreak3DConfig(steps=20))
    assert a == b and "steps" not in a and "t_end" not in a


def test_obstacle_box_stands_in_for_obstacle_fields():
    from tensorsph_b200.engine import obstacle_case
    cfg, box = obstacle_case(dx=0.05, steps=10)
    fp = ck.checkpoint_fingerprint(cfg, box)
    lo, hi = box
    assert fp["obstacle_x"] == lo[0] and fp["obstacle_z"] == lo[2]
    assert fp["obstacle_length"] == pytest.approx(hi[0] - lo[0])
    assert fp["obstacle_height"] == pytest.approx(hi[1] - lo[1])
    assert fp["obstacle_width"] == pytest.approx(hi[2] - lo[2])
    assert "obstacle_x" not in ck.checkpoint_fingerprint(cfg)
    # a run with the obstacle moved does not resume from this one's file
    moved = ((lo[0] + 0.1, lo[1], lo[2]), (hi[0] + 0.1, hi[1], hi[2]))
    assert ck.checkpoint_fingerprint(cfg, moved) != fp


def test_failed_write_keeps_previous_checkpoint(tmp_path, monkeypatch):
    cfg = types.SimpleNamespace(dx=0.1, dt=1e-3)
    run = types.SimpleNamespace(times=[0.0], front=[1.0], sph_impulse=[0.0] * 3, clamp_impulse=[0.0] * 3)
    path = tmp_path / "state.pt"
    common = dict(elapsed=0.1, dt=1e-3, positions=torch.zeros((3, 3), dtype=torch.float64),
                  velocity=torch.zeros((3, 3), dtype=torch.float64), run=run, speeds=0.0,
                  compression=0.0, escapes=0, clamps=0)
    ck.save_checkpoint(path, cfg, step=4, **common)
    real = torch.save

    def dying(obj, f, *a, **k):
        with open(f, "wb") as fh:  # a partial file, then the "crash"
            fh.write(b"PK\x03\x04truncated")
        raise OSError("killed while writing")

    monkeypatch.setattr(ck.torch, "save", dying)
    with pytest.raises(OSError):
        ck.save_checkpoint(path, cfg, step=9, **common)
    monkeypatch.setattr(ck.torch, "save", real)
    assert ck.load_checkpoint(path, cfg)["step"] == 4


def test_run_case_refuses_foreign_checkpoints(tmp_path):
    """Refusals happen before the engine is built: another configuration,
    another particle count, a file without this engine's run record (written
    by another driver) and a checkpoint at or past the run's last step."""
    from dataclasses import replace
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig
    from tensorsph_b200.engine import dam_break_3d_host_state, run_case
    cfg = DamBreak3DConfig(dx=0.04, pool_width=0.4, tank_depth=0.2, tank_height=0.4, column_width=0.2,
                           column_depth=0.2, column_height=0.2, steps=10)
    x = dam_break_3d_host_state(cfg)[0]
    run = types.SimpleNamespace(times=[0.0], front=[0.2], sph_impulse=[0.0] * 3, clamp_impulse=[0.0] * 3)
    common = dict(step=3, elapsed=4 * cfg.dt, dt=cfg.dt, positions=x, velocity=torch.zeros_like(x), run=run,
                  speeds=0.0, compression=0.0, escapes=0, clamps=0)
    mine = {"device_run": {}}
    path = tmp_path / "state.pt"
    ck.save_checkpoint(path, cfg, **common)
    with pytest.raises(ValueError, match="no device run record"):
        run_case(cfg, checkpoint_path=path)
    ck.save_checkpoint(path, cfg, **dict(common, positions=x[:-1], velocity=torch.zeros_like(x[:-1])), extra=mine)
    with pytest.raises(ValueError, match="checkpoint holds"):
        run_case(cfg, checkpoint_path=path)
    ck.save_checkpoint(path, cfg, **common, extra=mine)
    with pytest.raises(ValueError, match="different configuration: dx"):
        run_case(replace(cfg, dx=0.05), checkpoint_path=path)
    ck.save_checkpoint(path, cfg, **dict(common, step=10), extra=mine)
    with pytest.raises(ValueError, match="not below"):
        run_case(cfg, checkpoint_path=path)


def test_resumed_record_equals_uninterrupted_record():
    """The run record of a resumed device run, assembled from the checkpoint
    (written after step 10) and the meter rows of steps 11..20 of the new
    engine (whose counters and impulses restart at its admission), equals the
    record assembled from all 21 rows of a run that went through."""
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig
    from tensorsph_b200.engine import DIAG_FIELDS, _DeviceRecord, _sample_steps
    cfg = DamBreak3DConfig(steps=20, output_every=4, dt=1e-3, tvc_every=3)
    g = torch.Generator().manual_seed(5)
    rows = torch.rand((21, len(DIAG_FIELDS)), generator=g, dtype=torch.float64)
    cum = (8, 9, 10, 14, 20, 21, 22, 23, 24)   # counters and impulses: running totals
    rows[:, [8, 9, 10]] = torch.randint(0, 3, (21, 3), generator=g).double()
    rows[:, cum] = rows[:, cum].cumsum(0)
    samples = _sample_steps(cfg.steps, cfg.output_every, cfg.dt)
    whole = _DeviceRecord(cfg, samples, 0, None, 100, 7.0).collect(rows, 20)
    saved = _DeviceRecord(cfg, samples, 0, None, 100, 7.0).payload(rows[:11], 10)
    prev = {k: v for k, v in saved.items() if k not in ("extra", "dt")}
    prev.update(saved["extra"])
    later = rows[11:].clone()
    later[:, cum] -= rows[10, cum]
    resumed = _DeviceRecord(cfg, samples, 11, prev, 100, -1.0)
    part = resumed.collect(later, 20)
    assert resumed.initial_energy == 7.0
    for k in ("times", "front", "kinetic_energy", "potential_energy", "speed_samples", "escapes", "clamps",
              "rebuilds", "speeds", "compression"):
        assert part[k] == whole[k], k
    assert [e["step"] for e in part["tvc_log"]] == [e["step"] for e in whole["tvc_log"]] == [3, 6, 9, 12, 15, 18]
    np.testing.assert_allclose(part["obstacle_force"], whole["obstacle_force"], rtol=0, atol=0)
    np.testing.assert_allclose(part["sph_impulse"], whole["sph_impulse"], rtol=1e-14)
    np.testing.assert_allclose(part["clamp_impulse"], whole["clamp_impulse"], rtol=1e-14)
    assert len(whole["obstacle_force"]) == 20 and len(whole["times"]) == 6


def test_resumed_adaptive_record_equals_uninterrupted_record():
    """The same for an adaptive run: samples are the output_every-th steps and
    the final one with their times from the rows (column 25), the step range
    from column 27 and the Courant peak from columns 26 and 1 over every row,
    and a checkpoint carries them (and the rebuild count) into the resumed
    record; its dt is next_dt's step after the checkpointed one."""
    from dataclasses import replace
    from tensorsph_b200.dam_break_3d import DamBreak3DConfig
    from tensorsph_b200.engine import DIAG_FIELDS, _AdaptiveRecord
    cfg = replace(DamBreak3DConfig(steps=12, output_every=4, dt=1e-3), adaptive_dt=True)
    final = 17
    g = torch.Generator().manual_seed(9)
    rows = torch.rand((final + 1, len(DIAG_FIELDS)), generator=g, dtype=torch.float64)
    cum = (8, 9, 10, 14, 20, 21, 22, 23, 24)
    rows[:, [8, 9, 10]] = torch.randint(0, 3, (final + 1, 3), generator=g).double()
    rows[:, cum] = rows[:, cum].cumsum(0)
    rows[:, 26] = 0.9e-3 * (1.0 + 0.1 * torch.rand(final + 1, generator=g, dtype=torch.float64))
    rows[:, 27] = rows[:, 26]
    rows[:, 25] = torch.cat((torch.zeros(1, dtype=torch.float64), rows[:-1, 26].cumsum(0)))
    whole = _AdaptiveRecord(cfg, 0, None, 100, 7.0).collect(rows, final, final=final)
    assert [t for t in whole["times"]] == [float(rows[k, 25]) for k in (0, 4, 8, 12, 16, 17)]
    assert whole["dt_min"] == float(rows[:, 27].min()) and whole["dt_max"] == float(rows[:, 27].max())
    h = cfg.h_factor * cfg.dx
    assert whole["courant"] == pytest.approx(float((rows[:, 26] * (cfg.sound_speed + rows[:, 1])).max()) / h,
                                             rel=1e-15)
    assert whole["rebuilds"] == int(rows[final, 10])
    assert len(whole["obstacle_force"]) == final
    saved = _AdaptiveRecord(cfg, 0, None, 100, 7.0).payload(rows[:11], 10, dt=4.5e-4)
    assert saved["dt"] == 4.5e-4
    prev = {k: v for k, v in saved.items() if k not in ("extra", "dt")}
    prev.update(saved["extra"])
    later = rows[11:].clone()
    later[:, cum] -= rows[10, cum]
    part = _AdaptiveRecord(cfg, 11, prev, 100, -1.0).collect(later, final, final=final)
    for k in ("times", "front", "kinetic_energy", "potential_energy", "speed_samples", "escapes", "clamps",
              "rebuilds", "speeds", "compression", "dt_min", "dt_max"):
        assert part[k] == whole[k], k
    assert part["courant"] == pytest.approx(whole["courant"], rel=1e-15)
    np.testing.assert_allclose(part["obstacle_force"], whole["obstacle_force"], rtol=0, atol=0)
    np.testing.assert_allclose(part["sph_impulse"], whole["sph_impulse"], rtol=1e-14)
