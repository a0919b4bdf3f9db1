"""Integrator and clamps on the GPU (in place, like the reference)."""
from __future__ import annotations

import ctypes

import torch

from . import _lib


def _params(pos, lo, hi, tolerance, obstacle=None):
    prm = _lib.ClampParams()
    prm.dim, prm.dtype, prm.n = pos.shape[1], _lib.dtype_code(pos.dtype), pos.shape[0]
    for k in range(pos.shape[1]):
        prm.lo[k], prm.hi[k] = float(lo[k]), float(hi[k])
    prm.tolerance = float(tolerance)
    if obstacle is not None:
        (olo, ohi, eps) = obstacle
        prm.has_obstacle = 1
        for k in range(3):
            prm.ob_lo[k], prm.ob_hi[k] = float(olo[k]), float(ohi[k])
        prm.ob_eps = float(eps)
    return prm


def euler_clamp(pos: torch.Tensor, vel: torch.Tensor, acc: torch.Tensor | None, dt: float,
                lo, hi, tolerance: float, obstacle=None, counters: torch.Tensor | None = None):
    """``v += dt a; x += dt v`` then the box (and obstacle) clamp, in place.

    ``counters`` (device int64[2]) accumulates escapes and obstacle clamps
    without a host read; pass ``None`` to skip counting.
    """
    if not (pos.is_cuda and vel.is_cuda and pos.is_contiguous() and vel.is_contiguous()):
        raise ValueError("euler_clamp works in place on contiguous CUDA tensors")
    prm = _params(pos, lo, hi, tolerance, obstacle)
    _lib.check(_lib.lib().tsph_euler_clamp(ctypes.byref(prm), pos.data_ptr(), vel.data_ptr(),
                                           _lib.ptr(acc), float(dt), _lib.ptr(counters),
                                           _lib.stream(pos.device)), "tsph_euler_clamp")


def clamp_box(pos: torch.Tensor, vel: torch.Tensor, lo, hi, tolerance: float,
              obstacle=None) -> int:
    """In-place clamp of ``pos``/``vel`` (any device); returns the escape count."""
    dev = _lib.cuda_device(pos)
    P = pos.detach().to(dev).contiguous()
    V = vel.detach().to(dev).contiguous()
    counters = torch.zeros(2, dtype=torch.long, device=dev)
    euler_clamp(P, V, None, 0.0, lo, hi, tolerance, obstacle, counters)
    if P.data_ptr() != pos.data_ptr():
        pos.copy_(P.to(pos.device))
    if V.data_ptr() != vel.data_ptr():
        vel.copy_(V.to(vel.device))
    host = counters.tolist()
    return int(host[0] + host[1]) if obstacle is not None else int(host[0])
