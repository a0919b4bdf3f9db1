"""Persistent cache of autotuning results.

The engine's autotuners (``engine.tune_single_case`` for one large case,
``ensemble.autotune`` for a batched ensemble) time the list skin, the pair
kernels' block size and their batch depth on the device.  Their choice
depends on the workload and the GPU, not on the run, so it is kept in a JSON
file keyed by (kind, dimension, particle count to three significant digits,
h / dx, the candidate set, GPU name) and reused by later runs.

The file is ``$TSPH_TUNING_CACHE`` when set, else
``~/.cache/tensorsph_b200/tuning.json``.  Writes go through a temporary file
and an atomic rename, so concurrent processes never read a torn file (the
last writer wins).
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

__all__ = ["cache_path", "tuning_key", "lookup", "store"]


def cache_path() -> Path:
    env = os.environ.get("TSPH_TUNING_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "tensorsph_b200" / "tuning.json"


def _sig3(n: int) -> int:
    if n <= 0:
        return 0
    e = int(math.floor(math.log10(n))) - 2
    return int(round(n / 10 ** e) * 10 ** e) if e > 0 else int(n)


def tuning_key(kind: str, *, dim: int, particles: int, h_over_dx: float, candidates: dict,
               gpu: str) -> str:
    cand = ",".join(f"{k}={list(v)}" for k, v in sorted(candidates.items()))
    return f"{kind}|dim={dim}|n={_sig3(int(particles))}|h/dx={h_over_dx:.4g}|{cand}|gpu={gpu}"


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def lookup(key: str, path: Path | None = None):
    """The cached best configuration for ``key``, or None."""
    return _load(path or cache_path()).get(key)


def store(key: str, best: dict, path: Path | None = None) -> None:
    """Record ``best`` under ``key`` (atomic replace of the cache file)."""
    path = path or cache_path()
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        data = _load(path)
        data[key] = best
        tmp = path.with_suffix(f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home: tuning still works, it is just not kept
