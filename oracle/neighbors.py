"""Oracle: linked-cell pair search, periodic search, skin cache (numpy).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, with an independent per-cell loop, the reference functions

* ``brute_force_pairs``        -- src/tensorsph/neighbor_search.py:29-41
* ``cell_linked_pairs``        -- src/tensorsph/neighbor_search.py:44-120
* ``PairListCache``            -- src/tensorsph/neighbor_search.py:166-227
* ``periodic_pairs``           -- src/tensorsph/threed/neighbors3.py:71-142
* ``minimum_image``            -- src/tensorsph/threed/neighbors3.py:45-53

Arithmetic rules that make the integer output bit-exact with the reference:

* cell index ``floor(x / cutoff)`` by IEEE true division in the position dtype
  (``neighbor_search.py:63-64``);
* grid origin = per-axis minimum cell, row-major keys with the last axis
  fastest (``neighbor_search.py:65-72``);
* cell order is a *stable* sort by key (``neighbor_search.py:76-78``);
* squared distance summed sequentially ``((dx^2 + dy^2) + dz^2)`` in the
  dtype, compared with ``cutoff**2`` rounded to the dtype
  (``neighbor_search.py:113-114``).
"""
from __future__ import annotations

from itertools import product
import math

import numpy as np


def _check(pos, cutoff):
    pos = np.asarray(pos)
    if pos.ndim != 2:
        raise ValueError("positions must have shape (particle_count, dimension)")
    if not np.issubdtype(pos.dtype, np.floating):
        raise TypeError("positions must use a floating-point dtype")
    if not np.isfinite(pos).all():
        raise ValueError("positions must contain only finite values")
    if not math.isfinite(float(cutoff)) or cutoff <= 0:
        raise ValueError("cutoff must be finite and positive")
    return pos


def _empty():
    return np.zeros((0, 2), dtype=np.int64)


def squared_distance(delta):
    """``sum_k delta_k^2`` accumulated left to right in the dtype of ``delta``."""
    acc = delta[..., 0] * delta[..., 0]
    for axis in range(1, delta.shape[-1]):
        acc = acc + delta[..., axis] * delta[..., axis]
    return acc


def _finish(ii, jj):
    if not ii:
        return _empty()
    i = np.concatenate(ii)
    j = np.concatenate(jj)
    if i.size == 0:
        return _empty()
    order = np.lexsort((j, i))
    return np.stack((i[order], j[order]), axis=1).astype(np.int64)


def brute_force_pairs(pos, cutoff):
    pos = _check(pos, cutoff)
    n = pos.shape[0]
    if n < 2:
        return _empty()
    c2 = pos.dtype.type(float(cutoff) ** 2)
    ii, jj = [], []
    for a in range(n - 1):
        d2 = squared_distance(pos[a] - pos[a + 1:])
        hit = np.nonzero(d2 <= c2)[0] + a + 1
        ii.append(np.full(hit.size, a, dtype=np.int64))
        jj.append(hit.astype(np.int64))
    return _finish(ii, jj)


def cell_grid(pos, cutoff):
    """Cell coordinates, keys, extent and the stable cell order of a cloud."""
    dt = pos.dtype.type
    cells = np.floor(pos / dt(float(cutoff))).astype(np.int64)
    cells = cells - cells.min(axis=0)
    extent = cells.max(axis=0) + 1
    dim = pos.shape[1]
    strides = np.ones(dim, dtype=np.int64)
    for axis in range(dim - 2, -1, -1):
        strides[axis] = strides[axis + 1] * extent[axis + 1]
    keys = cells @ strides
    order = np.argsort(keys, kind="stable")
    return cells, keys, extent, strides, order


def cell_linked_pairs(pos, cutoff):
    pos = _check(pos, cutoff)
    n, dim = pos.shape
    if n < 2:
        return _empty()
    cells, keys, extent, strides, order = cell_grid(pos, cutoff)
    members: dict[tuple, np.ndarray] = {}
    sorted_keys = keys[order]
    boundaries = np.flatnonzero(np.diff(sorted_keys)) + 1
    for run in np.split(order, boundaries):
        members[tuple(cells[run[0]])] = run
    c2 = pos.dtype.type(float(cutoff) ** 2)
    offsets = list(product((-1, 0, 1), repeat=dim))
    ii, jj = [], []
    for key, mine in members.items():
        for off in offsets:
            other = members.get(tuple(k + d for k, d in zip(key, off)))
            if other is None:
                continue
            d2 = squared_distance(pos[mine][:, None, :] - pos[other][None, :, :])
            keep = (mine[:, None] < other[None, :]) & (d2 <= c2)
            a, b = np.nonzero(keep)
            ii.append(mine[a])
            jj.append(other[b])
    return _finish(ii, jj)


def minimum_image(delta, box):
    box = np.broadcast_to(np.asarray(box, dtype=delta.dtype).reshape(-1),
                          (delta.shape[-1],)).astype(delta.dtype)
    return delta - box * np.round(delta / box)


def periodic_grid(pos, box, cutoff):
    dim = pos.shape[1]
    dt = pos.dtype.type
    box_t = np.broadcast_to(np.asarray(box, dtype=pos.dtype).reshape(-1), (dim,))
    ncell = np.maximum(np.floor(box_t / dt(float(cutoff))).astype(np.int64), 3)
    width = box_t / ncell.astype(pos.dtype)
    cells = np.mod(np.floor(pos / width).astype(np.int64), ncell)
    strides = np.ones(dim, dtype=np.int64)
    for axis in range(dim - 2, -1, -1):
        strides[axis] = strides[axis + 1] * ncell[axis + 1]
    keys = cells @ strides
    order = np.argsort(keys, kind="stable")
    return cells, keys, ncell, box_t, order


def periodic_pairs(pos, box, cutoff):
    pos = np.asarray(pos)
    if pos.ndim != 2:
        raise ValueError("positions must be (N, D)")
    n, dim = pos.shape
    if n < 2:
        return _empty()
    if not np.isfinite(pos).all():
        raise ValueError("positions must be finite")
    cells, keys, ncell, box_t, order = periodic_grid(pos, box, cutoff)
    members: dict[tuple, np.ndarray] = {}
    sorted_keys = keys[order]
    for run in np.split(order, np.flatnonzero(np.diff(sorted_keys)) + 1):
        members[tuple(cells[run[0]])] = run
    c2 = pos.dtype.type(float(cutoff) ** 2)
    ii, jj = [], []
    for key, mine in members.items():
        for off in product((-1, 0, 1), repeat=dim):
            nk = tuple(int((k + d) % m) for k, d, m in zip(key, off, ncell))
            other = members.get(nk)
            if other is None:
                continue
            delta = minimum_image(pos[mine][:, None, :] - pos[other][None, :, :], box_t)
            keep = (mine[:, None] < other[None, :]) & (squared_distance(delta) <= c2)
            a, b = np.nonzero(keep)
            ii.append(mine[a])
            jj.append(other[b])
    return _finish(ii, jj)


class PairListCache:
    """Verlet-skin reuse, ``neighbor_search.py:166-227``."""

    def __init__(self, cutoff, skin, fluid_count=None):
        if not math.isfinite(float(cutoff)) or cutoff <= 0:
            raise ValueError("cutoff must be finite and positive")
        if not math.isfinite(float(skin)) or skin < 0:
            raise ValueError("skin must be finite and non-negative")
        if fluid_count is not None and fluid_count < 0:
            raise ValueError("fluid_count must be non-negative")
        self.cutoff, self.skin, self.fluid_count = float(cutoff), float(skin), fluid_count
        self._pairs = None
        self._anchor = None
        self.rebuilds = self.reuses = self.pruned = 0

    def displacement(self, pos):
        if self._anchor is None or self._anchor.shape != pos.shape:
            return float("inf")
        d = pos - self._anchor
        return float(np.sqrt(squared_distance(d)).max())

    def get(self, pos):
        if self._pairs is None or self.displacement(pos) > 0.5 * self.skin:
            pairs = cell_linked_pairs(pos, self.cutoff + self.skin)
            if self.fluid_count is not None and pairs.size:
                keep = (pairs[:, 0] < self.fluid_count) | (pairs[:, 1] < self.fluid_count)
                self.pruned += int(keep.size - keep.sum())
                pairs = pairs[keep]
            self._pairs = pairs
            self._anchor = pos.copy()
            self.rebuilds += 1
            return pairs, True
        self.reuses += 1
        return self._pairs, False


def cell_linked_pairs_batched(pos, cutoff):
    """Same pairs as :func:`cell_linked_pairs`, candidate expansion done in one
    batched pass (the structure of neighbor_search.py:80-120: every particle
    queries its 3^D neighbour cells through a sorted key table).  Used where
    the oracle has to run at tens of thousands of particles (CPU baseline)."""
    pos = _check(pos, cutoff)
    n, dim = pos.shape
    if n < 2:
        return _empty()
    cells, keys, extent, strides, order = cell_grid(pos, cutoff)
    sorted_keys = keys[order]
    uniq, first = np.unique(sorted_keys, return_index=True)
    counts = np.diff(np.append(first, n))
    c2 = pos.dtype.type(float(cutoff) ** 2)
    ii, jj = [], []
    for off in product((-1, 0, 1), repeat=dim):
        nb = cells + np.asarray(off, dtype=np.int64)
        inside = np.all((nb >= 0) & (nb < extent), axis=1)
        nkey = nb @ strides
        slot = np.clip(np.searchsorted(uniq, nkey), 0, uniq.size - 1)
        found = inside & (uniq[slot] == nkey)
        src = np.nonzero(found)[0]
        if src.size == 0:
            continue
        occ = counts[slot[src]]
        starts = first[slot[src]]
        rep = np.repeat(src, occ)
        within = np.arange(occ.sum()) - np.repeat(np.cumsum(occ) - occ, occ)
        j = order[np.repeat(starts, occ) + within]
        keep = rep < j
        rep, j = rep[keep], j[keep]
        d2 = squared_distance(pos[rep] - pos[j])
        keep = d2 <= c2
        ii.append(rep[keep])
        jj.append(j[keep])
    return _finish(ii, jj)
