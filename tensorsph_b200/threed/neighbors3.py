"""Periodic and open 3-D pair search (``tensorsph.threed.neighbors3``) on the GPU.

``periodic_pairs`` wraps cell indices with ``ncell = max(3, floor(L / cutoff))``
per axis and filters by the minimum-image distance, exactly like
threed/neighbors3.py:71-142; the work runs in ``csrc/cells.cu``.
"""
from __future__ import annotations

import torch

from .. import _lib
from ..neighbor_search import cell_linked_pairs, grid_pairs

__all__ = ["box_pairs", "periodic_pairs", "minimum_image"]


def box_pairs(positions: torch.Tensor, cutoff: float) -> torch.Tensor:
    return cell_linked_pairs(positions, cutoff)


def _box_list(box, dim):
    vals = torch.as_tensor(box, dtype=torch.float64).reshape(-1).tolist()
    if len(vals) == 1:
        vals = vals * dim
    if len(vals) != dim:
        raise ValueError(f"box must have 1 or {dim} edges, got {len(vals)}")
    return vals


def minimum_image(delta: torch.Tensor, box) -> torch.Tensor:
    """``delta - L round(delta / L)`` per axis."""
    box_t = torch.as_tensor(_box_list(box, delta.shape[-1]), dtype=delta.dtype,
                            device=delta.device).reshape(1, -1)
    return delta - box_t * torch.round(delta / box_t)


def periodic_pairs(positions: torch.Tensor, box, cutoff: float) -> torch.Tensor:
    if positions.dim() != 2:
        raise ValueError("positions must be (N, D)")
    n, dim = positions.shape
    if n < 2:
        return torch.zeros((0, 2), dtype=torch.int64, device=positions.device)
    vals = _box_list(box, dim)
    if any(b <= 0.0 for b in vals):
        raise ValueError("box edges must be positive")
    if dim > 3:
        raise ValueError("the CUDA search supports 1, 2 or 3 spatial dimensions")
    dev = _lib.cuda_device(positions)
    pos = _lib.to_dev(positions.detach(), dev)
    _lib.dtype_code(pos.dtype)
    pairs, _, _ = grid_pairs(pos, cutoff, box=vals)
    return pairs.to(positions.device)
