"""Drop-in linked-cell pair search on the B200 (``tensorsph.neighbor_search``).

Same names, arguments, return contract and exceptions as the reference module
(neighbor_search.py:9-227): unordered pairs ``(i, j)``, ``i < j``, sorted
lexicographically, as a ``(P, 2)`` int64 tensor on the input's device.

What runs underneath is the CUDA path of ``csrc/cells.cu``: integer cell keys,
a stable radix (counting) sort by key, a cell-run table and one candidate scan
per particle that counts, then emits, its row of partners, rows sorted in
registers/shared memory.  Results are bit-identical to the reference (same
cell arithmetic, same distance filter), which the GPU tests check against the
committed reference fixtures.
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib

__all__ = ["brute_force_pairs", "cell_linked_pairs", "cell_order", "PairListCache",
           "grid_pairs"]


def _validate(positions, cutoff):
    if not isinstance(positions, torch.Tensor):
        raise TypeError("positions must be a torch.Tensor")
    if positions.ndim != 2:
        raise ValueError("positions must have shape (particle_count, dimension)")
    if positions.shape[1] < 1:
        raise ValueError("positions must have at least one spatial dimension")
    if not positions.is_floating_point():
        raise TypeError("positions must use a floating-point dtype")
    if positions.shape[1] > 3:
        raise ValueError("the CUDA search supports 1, 2 or 3 spatial dimensions")
    if not math.isfinite(float(cutoff)) or cutoff <= 0:
        raise ValueError("cutoff must be finite and positive")
    return int(positions.shape[0]), int(positions.shape[1])


def _empty(device):
    return torch.empty((0, 2), dtype=torch.long, device=device)


def _plan(pos, cutoff, box=None):
    L = _lib.lib()
    dev = pos.device
    scratch = _lib.workspace(L.tsph_grid_plan_scratch_bytes(), dev)
    grid = _lib.Grid()
    box_arr = None
    if box is not None:
        box_arr = (ctypes.c_double * 3)(*([float(b) for b in box] + [1.0] * (3 - len(box))))
    rc = L.tsph_grid_plan(pos.data_ptr(), pos.shape[0], pos.shape[1], _lib.dtype_code(pos.dtype),
                          float(cutoff), box_arr, scratch.data_ptr(), ctypes.byref(grid),
                          _lib.stream(dev))
    if rc == _lib.ERR_NONFINITE:
        raise ValueError("positions must contain only finite values")
    _lib.check(rc, "tsph_grid_plan")
    ws = _lib.workspace(grid.workspace_bytes, dev)
    return grid, ws


def grid_pairs(pos: torch.Tensor, cutoff: float, box=None, row_limit: int | None = None,
               with_order: bool = False):
    """Pairs of a CUDA-resident cloud; returns ``(pairs, total, order)``.

    ``row_limit`` keeps only pairs whose first index is below it (the
    ``fluid_count`` pruning); ``total`` is the unpruned count.
    """
    L = _lib.lib()
    dev = pos.device
    n = pos.shape[0]
    grid, ws = _plan(pos, cutoff, box)
    order = torch.empty(n, dtype=torch.long, device=dev) if with_order else None
    s = _lib.stream(dev)
    _lib.check(L.tsph_grid_build(pos.data_ptr(), ctypes.byref(grid), ws.data_ptr(), ws.numel(),
                                 _lib.ptr(order), s), "tsph_grid_build")
    limit = n if row_limit is None else max(0, min(int(row_limit), n))
    kept, total = ctypes.c_int64(0), ctypes.c_int64(0)
    _lib.check(L.tsph_pairs_count(pos.data_ptr(), ctypes.byref(grid), limit, ws.data_ptr(),
                                  ws.numel(), ctypes.byref(kept), ctypes.byref(total), s),
               "tsph_pairs_count")
    pairs = torch.empty((kept.value, 2), dtype=torch.long, device=dev)
    if kept.value:
        ews = _lib.workspace(L.tsph_pairs_emit_workspace_bytes(kept.value, n), dev)
        _lib.check(L.tsph_pairs_emit(pos.data_ptr(), ctypes.byref(grid), limit, ws.data_ptr(),
                                     ws.numel(), ews.data_ptr(), ews.numel(), pairs.data_ptr(),
                                     kept.value, s), "tsph_pairs_emit")
    return pairs, int(total.value), order


def cell_linked_pairs(positions: torch.Tensor, cutoff: float) -> torch.Tensor:
    """Exact unordered pairs within ``cutoff`` (neighbor_search.py:44-120)."""
    n, _ = _validate(positions, cutoff)
    if n < 2:
        if n and not torch.isfinite(positions).all():
            raise ValueError("positions must contain only finite values")
        return _empty(positions.device)
    dev = _lib.cuda_device(positions)
    pos = _lib.to_dev(positions.detach(), dev)
    _lib.dtype_code(pos.dtype)
    pairs, _, _ = grid_pairs(pos, cutoff)
    return pairs.to(positions.device)


def cell_order(positions: torch.Tensor, cutoff: float) -> torch.Tensor:
    """Stable cell order of the cloud (the reference's ``argsort(inverse, stable=True)``)."""
    _validate(positions, cutoff)
    dev = _lib.cuda_device(positions)
    pos = _lib.to_dev(positions.detach(), dev)
    L = _lib.lib()
    grid, ws = _plan(pos, cutoff)
    order = torch.empty(pos.shape[0], dtype=torch.long, device=dev)
    _lib.check(L.tsph_grid_build(pos.data_ptr(), ctypes.byref(grid), ws.data_ptr(), ws.numel(),
                                 order.data_ptr(), _lib.stream(dev)), "tsph_grid_build")
    return order


def brute_force_pairs(positions: torch.Tensor, cutoff: float) -> torch.Tensor:
    """O(N^2) reference search on the GPU (neighbor_search.py:29-41)."""
    n, dim = _validate(positions, cutoff)
    if n and not torch.isfinite(positions).all():
        raise ValueError("positions must contain only finite values")
    if n < 2:
        return _empty(positions.device)
    dev = _lib.cuda_device(positions)
    pos = _lib.to_dev(positions.detach(), dev)
    L = _lib.lib()
    code = _lib.dtype_code(pos.dtype)
    ws = _lib.workspace(L.tsph_brute_workspace_bytes(n), dev)
    s = _lib.stream(dev)
    count = ctypes.c_int64(0)
    _lib.check(L.tsph_brute_pairs_count(pos.data_ptr(), n, dim, code, float(cutoff),
                                        ws.data_ptr(), ws.numel(), ctypes.byref(count), s),
               "tsph_brute_pairs_count")
    pairs = torch.empty((count.value, 2), dtype=torch.long, device=dev)
    if count.value:
        _lib.check(L.tsph_brute_pairs_emit(pos.data_ptr(), n, dim, code, float(cutoff),
                                           ws.data_ptr(), ws.numel(), pairs.data_ptr(),
                                           count.value, s), "tsph_brute_pairs_emit")
    return pairs.to(positions.device)


def max_displacement(positions: torch.Tensor, anchor: torch.Tensor, box=None) -> torch.Tensor:
    """Device scalar ``max |x - anchor|`` (minimum image when ``box`` is given)."""
    dev = positions.device
    out = torch.empty((), dtype=torch.float64, device=dev)
    L = _lib.lib()
    box_arr = None
    if box is not None:
        vals = [float(b) for b in (box if hasattr(box, "__len__") else [box] * positions.shape[1])]
        box_arr = (ctypes.c_double * 3)(*(vals + [1.0] * (3 - len(vals))))
    _lib.check(L.tsph_max_displacement(positions.data_ptr(), anchor.data_ptr(),
                                       positions.shape[0], positions.shape[1],
                                       _lib.dtype_code(positions.dtype), box_arr, out.data_ptr(),
                                       _lib.stream(dev)), "tsph_max_displacement")
    return out


class PairListCache:
    """Verlet-skin reuse of an inflated pair list (neighbor_search.py:166-227).

    The anchor positions stay on the GPU; the displacement test is one
    reduction kernel.  ``get`` still hands back a Python ``bool`` (the
    reference's contract), which is the single host read per step.
    """

    def __init__(self, cutoff: float, skin: float, fluid_count: int | None = None):
        if not math.isfinite(float(cutoff)) or cutoff <= 0:
            raise ValueError("cutoff must be finite and positive")
        if not math.isfinite(float(skin)) or skin < 0:
            raise ValueError("skin must be finite and non-negative")
        if fluid_count is not None and fluid_count < 0:
            raise ValueError("fluid_count must be non-negative")
        self.cutoff = float(cutoff)
        self.skin = float(skin)
        self.fluid_count = fluid_count
        self._pairs: torch.Tensor | None = None
        self._anchor: torch.Tensor | None = None
        self.rebuilds = 0
        self.reuses = 0
        self.pruned = 0

    def displacement(self, positions: torch.Tensor) -> float:
        if self._anchor is None or self._anchor.shape != positions.shape:
            return float("inf")
        dev = self._anchor.device
        pos = _lib.to_dev(positions.detach(), dev, self._anchor.dtype)
        return float(max_displacement(pos, self._anchor))

    def _build(self, positions: torch.Tensor) -> torch.Tensor:
        _validate(positions, self.cutoff + self.skin)
        dev = _lib.cuda_device(positions)
        pos = _lib.to_dev(positions.detach(), dev)
        if pos.shape[0] < 2:
            if pos.shape[0] and not torch.isfinite(pos).all():
                raise ValueError("positions must contain only finite values")
            return _empty(positions.device)
        pairs, total, _ = grid_pairs(pos, self.cutoff + self.skin, row_limit=self.fluid_count)
        if self.fluid_count is not None:
            self.pruned += total - pairs.shape[0]
        return pairs.to(positions.device)

    def get(self, positions: torch.Tensor) -> tuple[torch.Tensor, bool]:
        """Return ``(pairs, rebuilt)`` for the current positions."""
        if self._pairs is None or self.displacement(positions) > 0.5 * self.skin:
            self._pairs = self._build(positions)
            dev = _lib.cuda_device(positions)
            self._anchor = positions.detach().to(dev).clone()
            self.rebuilds += 1
            return self._pairs, True
        self.reuses += 1
        return self._pairs, False
