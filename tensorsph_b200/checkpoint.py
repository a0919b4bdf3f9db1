"""Crash-safe run checkpoints in the format of the 3-D obstacle case
(kleefsman_obstacle_3d.py:477-546), written off the step loop.

The payload is the reference's: a ``torch.save`` dict with ``version`` 3, the
configuration ``fingerprint``, ``step``, ``elapsed``, ``dt``, CPU
``positions`` and ``velocity``, the sampled series (``times``, ``height``,
``local_h2``, ``front``, ``bypass`` and ``slab`` when the run has it), the
running maxima and counters (``speeds``, ``compression``, ``escapes``,
``clamps``) and both obstacle impulses.  The file is replaced atomically
(``tmp`` + ``os.replace``), so a process killed while writing leaves the
previous checkpoint or the new one, never a truncated file.  ``load_checkpoint``
refuses another version or a configuration whose fingerprint differs;
``t_end`` and the step count are not part of it (a run may resume with a
longer horizon).

``CheckpointWriter`` is the device side: it copies a case's positions,
velocities and meter rows to pinned host memory on a side stream and writes
the file on a background thread, so the step loop only pays for the read
kernel and never waits on the disk.
"""
from __future__ import annotations

import os
import threading
import time
from pathlib import Path

import torch

__all__ = ["CHECKPOINT_VERSION", "CHECKPOINT_FINGERPRINT_FIELDS", "checkpoint_fingerprint",
           "save_checkpoint", "load_checkpoint", "CheckpointWriter"]

CHECKPOINT_VERSION = 3

#: configuration fields that make a checkpoint of another run useless (the
#: reference's list and order: the fingerprint is part of the file format)
CHECKPOINT_FINGERPRINT_FIELDS = (
    "dx", "sound_speed", "gamma", "rho0", "h_factor", "wall_layers",
    "obstacle_z", "obstacle_width", "station_offset", "gauge_aperture",
    "arrival_threshold", "pair_skin_factor", "density_diffusion",
    "surface_pressure_closure", "adaptive_dt", "max_courant", "viscosity",
    "pool_width", "tank_depth", "tank_height", "column_width",
    "column_height", "column_depth", "obstacle_x", "obstacle_length",
    "obstacle_height", "gravity", "wall_friction", "dt", "output_every",
)


def _obstacle_fields(obstacle) -> dict:
    """The obstacle box ``(lo, hi)`` as the obstacle case's fields: upstream
    face x, spanwise start z, and the box's length, height and width."""
    lo, hi = obstacle
    return {"obstacle_x": float(lo[0]), "obstacle_z": float(lo[2]),
            "obstacle_length": float(hi[0]) - float(lo[0]),
            "obstacle_height": float(hi[1]) - float(lo[1]),
            "obstacle_width": float(hi[2]) - float(lo[2])}


def checkpoint_fingerprint(cfg, obstacle=None) -> dict:
    """The subset of ``cfg`` that decides whether a checkpoint is reusable.

    A configuration of the obstacle case carries every field; a 3-D dam-break
    configuration carries those it has, with the obstacle box ``(lo, hi)`` of
    a device run standing in for the obstacle fields."""
    have = _obstacle_fields(obstacle) if obstacle is not None else {}
    fields = {}
    for name in CHECKPOINT_FINGERPRINT_FIELDS:
        if hasattr(cfg, name):
            fields[name] = getattr(cfg, name)
        elif name in have:
            fields[name] = have[name]
    if getattr(cfg, "pressure_disk_diameter", 0.0):
        fields["pressure_disk_diameter"] = cfg.pressure_disk_diameter
    return fields


def _atomic_save(payload: dict, path: Path) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(path.name + ".tmp")
    torch.save(payload, tmp)
    os.replace(tmp, path)


def _payload(fingerprint, *, step, elapsed, dt, positions, velocity, run, speeds, compression,
             escapes, clamps) -> dict:
    payload = {
        "version": CHECKPOINT_VERSION,
        "fingerprint": fingerprint,
        "step": int(step),
        "elapsed": float(elapsed),
        "dt": float(dt),
        "positions": positions.detach().to("cpu").clone(),
        "velocity": velocity.detach().to("cpu").clone(),
        "times": list(run.times),
        "height": list(getattr(run, "height", [])),
        "local_h2": list(getattr(run, "local_h2", [])),
        "front": list(run.front),
        "bypass": list(getattr(run, "bypass", [])),
        "speeds": float(speeds),
        "compression": float(compression),
        "escapes": int(escapes),
        "clamps": int(clamps),
        "sph_impulse": list(run.sph_impulse), "clamp_impulse": list(run.clamp_impulse),
    }
    if hasattr(run, "slab"):
        payload["slab"] = list(run.slab)
    return payload


def save_checkpoint(path, cfg, *, step, elapsed, dt, positions, velocity, run, speeds, compression,
                    escapes, clamps, obstacle=None, extra: dict | None = None) -> None:
    """Write the integration state atomically (``tmp`` + ``os.replace``).

    ``run`` supplies ``times`` and ``front`` and, where it has them, the gauge
    series, ``sph_impulse`` and ``clamp_impulse``; ``extra`` adds keys of
    this engine's own next to the reference's."""
    payload = _payload(checkpoint_fingerprint(cfg, obstacle), step=step, elapsed=elapsed, dt=dt,
                       positions=positions, velocity=velocity, run=run, speeds=speeds,
                       compression=compression, escapes=escapes, clamps=clamps)
    if extra:
        payload.update(extra)
    _atomic_save(payload, Path(path))


def load_checkpoint(path, cfg, obstacle=None) -> dict:
    """Load a checkpoint, refusing one written for different physics."""
    payload = torch.load(path, map_location="cpu", weights_only=False)
    if payload.get("version") != CHECKPOINT_VERSION:
        raise ValueError(f"checkpoint version {payload.get('version')} != {CHECKPOINT_VERSION}")
    got = payload.get("fingerprint", {})
    want = checkpoint_fingerprint(cfg, obstacle)
    diff = {k: (got.get(k), want.get(k)) for k in got.keys() | want.keys() if got.get(k) != want.get(k)}
    if diff:
        raise ValueError("checkpoint was written for a different configuration: "
                         + ", ".join(f"{k}: {g!r} -> {w!r}" for k, (g, w) in sorted(diff.items())))
    return payload


class _Series:
    """The sampled series and impulses a payload takes from its run."""

    def __init__(self, times, front, sph_impulse, clamp_impulse):
        self.times, self.front = times, front
        self.sph_impulse, self.clamp_impulse = sph_impulse, clamp_impulse


class CheckpointWriter:
    """Asynchronous checkpoints of one engine case.

    ``take`` enqueues, on a side stream ordered after the engine's work so
    far, the read of the case's fluid state and meter rows and their copy to
    pinned host memory, then hands the rest to a writer thread: wait for the
    copies, assemble the payload (``assemble(rows)`` gives the series and
    maxima from the meter rows), write it atomically.  One write is in flight
    at a time; ``take`` waits for the previous one first, which bounds the
    pinned memory to one state.  ``close`` waits for the last write and
    re-raises a writer error."""

    def __init__(self, eng, case_id: int, path, cfg, *, obstacle=None):
        self.eng, self.case_id = eng, case_id
        self.path, self.cfg, self.obstacle = Path(path), cfg, obstacle
        self.side = torch.cuda.Stream(device=eng.device)
        self.thread: threading.Thread | None = None
        self.error: BaseException | None = None
        self.written = 0
        self.write_seconds: list[float] = []  # per file: copies awaited, payload built, written

    def take(self, step: int, elapsed: float, first_row: int, rows: int, assemble) -> None:
        """Checkpoint the state after the update of global step ``step``;
        ``rows`` meter rows from global step ``first_row`` go to ``assemble``."""
        from .engine import BatchEngine
        self.wait()
        with torch.cuda.stream(self.side):
            x, v, _, _ = self.eng.read(self.case_id)
            diag = BatchEngine.diagnostics(self.eng, self.case_id, first_row, rows)
            hx = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
            hv = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
            hd = torch.empty(diag.shape, dtype=diag.dtype, pin_memory=True)
            hx.copy_(x, non_blocking=True)
            hv.copy_(v, non_blocking=True)
            hd.copy_(diag, non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.side)

        def write():
            t0 = time.perf_counter()
            try:
                done.synchronize()
                info = assemble(hd)
                series = _Series(info["times"], info["front"], info["sph_impulse"], info["clamp_impulse"])
                save_checkpoint(self.path, self.cfg, step=step, elapsed=elapsed, dt=info["dt"],
                                positions=hx, velocity=hv, run=series, speeds=info["speeds"],
                                compression=info["compression"], escapes=info["escapes"],
                                clamps=info["clamps"], obstacle=self.obstacle, extra=info.get("extra"))
                self.written += 1
                self.write_seconds.append(time.perf_counter() - t0)
            except BaseException as exc:  # re-raised on the caller's thread
                self.error = exc

        self.thread = threading.Thread(target=write, name="tsph-checkpoint", daemon=True)
        self.thread.start()

    def wait(self) -> None:
        if self.thread is not None:
            self.thread.join()
            self.thread = None
        if self.error is not None:
            err, self.error = self.error, None
            raise err

    def close(self) -> None:
        self.wait()
