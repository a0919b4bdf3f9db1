"""Lind particle shifting on the GPU (``tensorsph.particle_shifting``).

``shift_positions`` keeps the reference signature and result
(particle_shifting.py:166-224): concentration ``C`` with the 2-D cubic
normalisation (as the reference applies it in every dimension), its
antisymmetric gradient, the free-surface detector against the 95th
percentile of ``C`` (a device radix select, linear interpolation like
``torch.quantile``), tangential projection and the ``limit * h`` cap -- all in
``csrc/shift.cu``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
import math

import torch

from . import _lib
from .droplet_impact import symmetric_rows
from .neighbor_search import grid_pairs

__all__ = ["ShiftingState", "shift_positions", "concentration", "estimate_reference_concentration"]


@dataclass
class ShiftingState:
    concentration: torch.Tensor
    grad_c: torch.Tensor
    normal: torch.Tensor
    shift: torch.Tensor
    free_surface: torch.Tensor
    c_reference: float
    magnitude: float
    clipped: float = 0.0
    extras: dict = field(default_factory=dict)

    @property
    def max_shift(self) -> float:
        return (float(torch.linalg.vector_norm(self.shift, dim=-1).max())
                if self.shift.numel() else 0.0)


def _run(pos, volume, h, magnitude, cap, free_surface, pairs, c_reference):
    n, dim = pos.shape
    dev = _lib.cuda_device(pos)
    dtype = pos.dtype
    P = _lib.to_dev(pos.detach(), dev)
    Vol = _lib.to_dev(volume.detach(), dev, dtype)
    if pairs is None:
        pairs_dev, _, _ = grid_pairs(P, 2.0 * h) if n >= 2 else (
            torch.zeros((0, 2), dtype=torch.long, device=dev), 0, None)
    else:
        pairs_dev = _lib.to_dev(pairs, dev)
    rowptr, entries = symmetric_rows(pairs_dev, n)
    prm = _lib.ShiftParams()
    prm.dim, prm.dtype, prm.n = dim, _lib.dtype_code(dtype), n
    prm.h, prm.sigma = float(h), 10.0 / (7.0 * math.pi * h * h)
    prm.magnitude, prm.cap, prm.free_surface = magnitude, cap, float(free_surface)
    prm.c_reference = -1.0 if c_reference is None else float(c_reference)
    out = torch.empty_like(P)
    c = torch.empty(n, dtype=dtype, device=dev)
    grad = torch.empty_like(P)
    normal = torch.empty_like(P)
    shift = torch.empty_like(P)
    fs = torch.empty(n, dtype=torch.uint8, device=dev)
    cref = torch.zeros((), dtype=torch.float64, device=dev)
    io = _lib.ShiftIO(P.data_ptr(), Vol.data_ptr(), rowptr.data_ptr(), entries.data_ptr(),
                      out.data_ptr(), c.data_ptr(), grad.data_ptr(), normal.data_ptr(),
                      shift.data_ptr(), fs.data_ptr(), cref.data_ptr())
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_shift_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_shift_positions(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(),
                                      ws.numel(), _lib.stream(dev)), "tsph_shift_positions")
    return out, c, grad, normal, shift, fs.bool(), cref


def concentration(pos, volume, h, pairs=None):
    if pos.ndim != 2 or volume.shape != pos.shape[:1]:
        raise ValueError("pos must be (N, D) and volume must be (N,)")
    if not math.isfinite(h) or h <= 0:
        raise ValueError("h must be finite and positive")
    _, c, *_ = _run(pos, volume, h, 0.0, 0.0, 0.95, pairs, 1.0)
    return c.to(pos.device)


def estimate_reference_concentration(c: torch.Tensor, percentile: float = 95.0) -> float:
    if c.numel() == 0:
        return 0.0
    q = min(max(percentile, 0.0), 100.0) / 100.0
    dev = _lib.cuda_device(c)
    x = _lib.to_dev(c.detach(), dev)
    out = torch.empty((), dtype=torch.float64, device=dev)
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_quantile_workspace_bytes(x.numel()), dev)
    _lib.check(L.tsph_quantile(x.data_ptr(), x.numel(), _lib.dtype_code(x.dtype), q,
                               out.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(dev)),
               "tsph_quantile")
    return float(out)


def shift_positions(pos, volume, h, *, dt, v_ref, strength=1.0, limit=0.25, free_surface=0.95,
                    pairs=None, c_reference=None, return_state=False):
    """One shifting pass; returns the shifted positions (and the state)."""
    if pos.ndim != 2 or volume.shape != pos.shape[:1]:
        raise ValueError("pos must be (N, D) and volume must be (N,)")
    if dt <= 0 or not math.isfinite(dt):
        raise ValueError("dt must be finite and positive")
    n = pos.shape[0]
    if n == 0:
        return pos.clone() if not return_state else (pos.clone(), None)
    magnitude = float(strength) * h * float(v_ref) * float(dt)
    cap = float(limit) * h
    out, c, grad, normal, shift, fs, cref = _run(pos, volume, h, magnitude, cap, free_surface,
                                                 pairs, c_reference)
    dev = pos.device
    if not return_state:
        return out.to(dev)
    mag = torch.linalg.vector_norm(shift, dim=-1)
    clipped = float((torch.isclose(mag, torch.full_like(mag, cap))).double().mean())
    return out.to(dev), ShiftingState(
        concentration=c.to(dev), grad_c=grad.to(dev), normal=normal.to(dev), shift=shift.to(dev),
        free_surface=fs.to(dev), c_reference=float(cref), magnitude=magnitude, clipped=clipped)
