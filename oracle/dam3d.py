"""Oracle: the 3-D dam-break step loop with a box obstacle, in FP64 numpy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the FP64 side that the
device engine's FP32-pair run is compared with, field by field.

One step, as the reference's loops take it:

* ``rhs_3d`` with the obstacle reaction (dam_break_3d.py:290-422), on the pairs
  of a ``PairListCache`` at 2h + skin built over fluid + walls and pruned of
  wall-wall pairs (neighbor_search.py:166-227; pairs between 2h and 2h + skin
  add exactly zero);
* semi-implicit Euler v += dt a, x += dt v and the box clamp
  ``apply_boundary_3d`` (dam_break_3d.py:429-452, tolerance 0.25 dx);
* the obstacle clamp ``clamp_out_of_obstacle`` (kleefsman_obstacle_3d.py:208-266):
  a particle inside the box goes to its nearest face plus 0.01 dx and loses
  the normal velocity;
* from the second step on, every ``shift_every`` steps, Lind shifting of the
  clamped positions with volumes m / rho of this step and v_ref = max(speed
  at the start of the step, 0.05 c0) (the shifting hook of dam_break.py:424-433,
  ``shift_positions`` particle_shifting.py:166-224 on fresh 2h pairs).

Each step records what the reference loops report: the fluid density and
pressure, the acceleration, the summed obstacle force
(kleefsman_obstacle_3d.py:649-653) and the front, max x of the fluid
(``front_position_3d``, dam_break_3d.py:459-463), at the start of the step.
"""
from __future__ import annotations

import numpy as np

from . import neighbors as on
from . import pairpass as op


def obstacle_clamp(x, v, lo, hi, dx):
    """clamp_out_of_obstacle (kleefsman_obstacle_3d.py:208-266), in place."""
    inside = np.all((x > lo) & (x < hi), axis=1)
    for a in np.nonzero(inside)[0]:
        cand = [x[a, 0] - lo[0], hi[0] - x[a, 0], x[a, 1] - lo[1], hi[1] - x[a, 1],
                x[a, 2] - lo[2], hi[2] - x[a, 2]]
        f = int(np.argmin(cand))
        k = f // 2
        x[a, k] = hi[k] + 0.01 * dx if f % 2 else lo[k] - 0.01 * dx
        v[a, k] = 0.0
    return int(inside.sum())


def run(cfg, obstacle, x, mass, wall, n_ob, steps, *, shift_every=0, skin=None, record=True,
        v0=None, first_step=0):
    """FP64 trajectory of ``steps`` steps from positions ``x`` and velocities
    ``v0`` (rest when None); ``first_step`` numbers the first step (the shifting
    cadence counts from it).  Returns ``(records, x, v)``: per step a dict of
    ``rho``, ``p``, ``acc`` (fluid), ``force`` (obstacle, summed) and ``front``,
    or an empty list when ``record`` is false."""
    x = np.array(x, dtype=np.float64)
    mass = np.asarray(mass, dtype=np.float64)
    wall = np.asarray(wall, dtype=np.float64)
    v = np.zeros_like(x) if v0 is None else np.array(v0, dtype=np.float64)
    n = x.shape[0]
    h = cfg.h_factor * cfg.dx
    skin = cfg.pair_skin_factor * h if skin is None else skin
    box = np.array([cfg.pool_width, cfg.tank_height, cfg.tank_depth])
    tol = 0.25 * cfg.dx
    lo = hi = None
    if obstacle is not None:
        lo, hi = np.asarray(obstacle[0], dtype=np.float64), np.asarray(obstacle[1], dtype=np.float64)
    anchor, pairs = None, None
    out = []
    for step in range(first_step, first_step + steps):
        if anchor is None or np.sqrt(((x - anchor) ** 2).sum(1)).max() > 0.5 * skin:
            pairs = on.cell_linked_pairs_batched(np.concatenate((x, wall)), 2.0 * h + skin)
            pairs = pairs[pairs[:, 0] < n]
            anchor = x.copy()
        rho, p, acc, react = op.rhs_3d(x, v, mass, cfg, pairs=pairs, wall=wall, dt=cfg.dt,
                                       return_wall_force=True)
        if record:
            out.append({"rho": rho, "p": p, "acc": acc,
                        "force": react[wall.shape[0] - n_ob:].sum(axis=0) if n_ob else np.zeros(3),
                        "front": float(x[:, 0].max()) if n else 0.0})
        speed = float(np.sqrt((v * v).sum(1)).max()) if n else 0.0
        v = v + cfg.dt * acc
        x = x + cfg.dt * v
        out_mask = (x < -tol) | (x > box + tol)
        x = np.clip(x, 0.0, box)
        v[out_mask] = 0.0
        if lo is not None:
            obstacle_clamp(x, v, lo, hi, cfg.dx)
        if shift_every and step > 0 and step % shift_every == 0:
            x, _ = op.shift_positions(x, mass / rho, h, dt=cfg.dt,
                                      v_ref=max(speed, 0.05 * cfg.sound_speed))
    return out, x, v
