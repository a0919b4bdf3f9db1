"""Device-resident 3-D dam-break engine (``csrc/engine.cu``) and its case drivers.

``DamBreak3DEngine`` owns one GPU-resident case: FP64 positions, velocities
and meters, cell-sorted particles, a skin-cached neighbour list rebuilt on the
device, and one CUDA graph per step (rebuild check, density, Molteni
diffusion, Tait, Adami walls, force, obstacle reaction, semi-implicit Euler
with the box and obstacle clamps, optional Lind shift).

``run_case`` is the drop-in for ``tensorsph.dam_break_3d.run_case``
(dam_break_3d.py:569-734) and returns the same ``DamBreak3DRun`` record;
``obstacle_case`` builds the 3-D dam break with a box obstacle of the
headline benchmark (fluid 1.2 x 1.0 x 0.55 m in a 3.2 x 1.0 x 1.0 m tank,
obstacle 0.16 x 0.16 x 0.4 m).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
import math

import torch

from . import _lib
from .dam_break_3d import DamBreak3DConfig, make_column_3d, mass_3d, wall_lattice_3d

__all__ = ["DamBreak3DEngine", "DamBreak3DRun", "obstacle_case", "obstacle_lattice_3d",
           "run_case", "DIAG_FIELDS"]

DIAG_FIELDS = ("rho_max", "speed_max", "front", "force_x", "force_y", "force_z", "kinetic",
               "potential", "escapes", "clamps", "rebuilds", "row_max", "step", "status",
               "impulse_x", "c_reference")


def obstacle_lattice_3d(lo, hi, dx: float) -> torch.Tensor:
    """Solid particles filling the box ``[lo, hi]`` on the fluid lattice
    (kleefsman_obstacle_3d.py:187-205)."""
    def span(a, b):
        n = max(1, int(round((b - a) / dx)))
        return a + (torch.arange(n, dtype=torch.float64) + 0.5) * dx
    gx, gy, gz = torch.meshgrid(span(lo[0], hi[0]), span(lo[1], hi[1]), span(lo[2], hi[2]),
                                indexing="xy")
    return torch.stack((gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)), dim=-1)


def clamp_out_of_obstacle_host(pos: torch.Tensor, lo, hi, eps: float) -> int:
    """Move fluid particles that start inside the obstacle out through the
    nearest face (set-up only, kleefsman_obstacle_3d.py:208-266)."""
    inside = torch.ones(pos.shape[0], dtype=torch.bool)
    for k in range(3):
        inside &= (pos[:, k] > lo[k]) & (pos[:, k] < hi[k])
    idx = inside.nonzero().reshape(-1)
    if idx.numel() == 0:
        return 0
    px = pos[idx]
    cand = torch.stack((px[:, 0] - lo[0], hi[0] - px[:, 0], px[:, 1] - lo[1], hi[1] - px[:, 1],
                        px[:, 2] - lo[2], hi[2] - px[:, 2]), dim=1)
    which = cand.argmin(dim=1)
    for f in range(6):
        k = f // 2
        sel = which == f
        px[sel, k] = (hi[k] + eps) if f % 2 else (lo[k] - eps)
    pos[idx] = px
    return int(idx.numel())


def obstacle_case(dx: float = 0.0069, *, viscosity: float = 1.0e-6, density_diffusion: float = 0.1,
                  steps: int = 5000, courant: float = 0.25):
    """Configuration and obstacle box of the 3-D dam break with an obstacle.

    Fluid block 1.2 x 1.0 x 0.55 m in a 3.2 x 1.0 x 1.0 m tank, three wall
    layers, Tait rho0 = 1000, gamma = 7, c0 = 10 sqrt(2 g 0.55), h = 1.3 dx,
    Molteni diffusion delta = 0.1, acoustic CFL 0.25.  The obstacle
    (0.16 streamwise x 0.16 high x 0.4 spanwise) stands on the floor, centred
    across the tank, its centre 0.744 m from the downstream wall.
    """
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 0.55)
    h = 1.3 * dx
    cfg = DamBreak3DConfig(dx=dx, pool_width=3.2, tank_depth=1.0, tank_height=1.0,
                           column_width=1.2, column_depth=1.0, column_height=0.55, wall_layers=3,
                           density_diffusion=density_diffusion, sound_speed=c0,
                           viscosity=viscosity, dt=courant * h / c0, max_courant=courant,
                           steps=steps)
    x0 = 3.2 - 0.744 - 0.08
    lo = (x0, 0.0, 0.3)
    hi = (x0 + 0.16, 0.16, 0.7)
    return cfg, (lo, hi)


@dataclass
class DamBreak3DRun:
    """Run record with the fields of the reference ``DamBreak3DRun`` that the
    engine measures (dam_break_3d.py:488-549) plus the obstacle force series."""

    times: list
    front: list
    kinetic_energy: list
    potential_energy: list
    mass: float
    escaped: int
    rebuilds: int
    max_speed: float
    max_density_compression: float
    initial_mass: float
    final_mass: float
    final_positions: torch.Tensor
    initial_energy: float = 0.0
    final_energy: float = 0.0
    steps_taken: int = 0
    simulated_time: float = 0.0
    obstacle_force: list = field(default_factory=list)
    obstacle_impulse: list = field(default_factory=list)
    obstacle_clamps: int = 0

    @property
    def mass_drift(self) -> float:
        return self.final_mass - self.initial_mass


class DamBreak3DEngine:
    """One device-resident 3-D dam-break case."""

    def __init__(self, cfg: DamBreak3DConfig, *, obstacle=None, shift_every: int = 0,
                 seed: int | None = None, max_neighbors: int = 160, diag_ring: int = 8192,
                 device: torch.device | None = None, host_state=None):
        dev = device or _lib.cuda_device()
        self.cfg = cfg
        self.device = dev
        self.stream = torch.cuda.Stream(device=dev)
        h = cfg.h_factor * cfg.dx
        if host_state is None:
            host_state = self.build_host_state(cfg, obstacle, seed)
        x, mass, wall, n_ob = host_state
        self.n_fluid, self.n_wall, self.n_obstacle = x.shape[0], wall.shape[0], n_ob
        prm = _lib.EngineParams()
        prm.n_fluid, prm.n_wall, prm.n_obstacle = self.n_fluid, self.n_wall, n_ob
        prm.max_neighbors, prm.shift_every, prm.diag_ring = max_neighbors, shift_every, diag_ring
        prm.has_obstacle = 1 if obstacle is not None else 0
        prm.dx, prm.h, prm.rho0 = cfg.dx, h, cfg.rho0
        prm.sound_speed, prm.gamma, prm.gravity = cfg.sound_speed, cfg.gamma, cfg.gravity
        prm.viscosity, prm.wall_friction = cfg.viscosity, cfg.wall_friction
        if cfg.density_diffusion > 0.0 and cfg.density_diffusion_form != "molteni":
            raise ValueError("the 3-D pass implements the 'molteni' diffusion form only")
        prm.diffusion_scale = (2.0 * cfg.density_diffusion * cfg.sound_speed * cfg.h_factor
                               * cfg.dx if cfg.density_diffusion > 0.0 else 0.0)
        prm.dt = cfg.dt
        prm.wall_mass = mass_3d(cfg.dx, cfg.h_factor, cfg.rho0, cfg.density_calibration)
        prm.skin = cfg.pair_skin_factor * h
        for k, v in enumerate((cfg.pool_width, cfg.tank_top(), cfg.tank_depth)):
            prm.box_hi[k] = v
        prm.tolerance = 0.25 * cfg.dx
        if obstacle is not None:
            for k in range(3):
                prm.ob_lo[k], prm.ob_hi[k] = obstacle[0][k], obstacle[1][k]
            prm.ob_eps = 0.01 * cfg.dx
        prm.shift_strength = getattr(cfg, "shift_strength", 1.0)
        prm.shift_limit = getattr(cfg, "shift_limit", 0.25)
        prm.shift_free_surface = 0.95
        prm.shift_vref_floor = 0.05 * cfg.sound_speed
        allpos = torch.cat((x, wall)) if self.n_wall else x
        lo = allpos.min(dim=0).values.tolist()
        hi = allpos.max(dim=0).values.tolist()
        for k in range(3):
            prm.grid_lo[k] = min(lo[k], 0.0) - 2.0 * cfg.dx
            prm.grid_hi[k] = max(hi[k], prm.box_hi[k]) + 2.0 * cfg.dx
        self.params = prm
        L = _lib.lib()
        nbytes = L.tsph_engine_bytes(ctypes.byref(prm))
        if nbytes <= 0:
            raise ValueError("invalid engine parameters")
        self._handle = ctypes.c_void_p(None)
        with torch.cuda.stream(self.stream):
            self.arena = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            X = x.to(dev, torch.float64, non_blocking=True).contiguous()
            V = torch.zeros_like(X)
            M = mass.to(dev, torch.float64, non_blocking=True).contiguous()
            Wl = wall.to(dev, torch.float64, non_blocking=True).contiguous()
            _lib.check(L.tsph_engine_create(ctypes.byref(prm), self.arena.data_ptr(), nbytes,
                                            X.data_ptr(), V.data_ptr(), M.data_ptr(),
                                            Wl.data_ptr() if self.n_wall else None,
                                            self.stream.cuda_stream, ctypes.byref(self._handle)),
                       "tsph_engine_create")
        self.initial_mass = float(mass.sum())
        self.initial_pe = float((mass * cfg.gravity * x[:, 1]).sum())
        self.steps_done = 0
        self.state_bytes = (X.numel() + M.numel() + Wl.numel()) * 8

    @staticmethod
    def build_host_state(cfg, obstacle=None, seed=None):
        """Host lattices of the case: fluid (FP64), masses, walls (+ obstacle last)."""
        saved = torch.get_default_dtype()
        torch.set_default_dtype(torch.float64)
        try:
            x, mass = make_column_3d(cfg, "cpu", seed=seed)
            wall = wall_lattice_3d(cfg, "cpu")
            n_ob = 0
            if obstacle is not None:
                ob = obstacle_lattice_3d(obstacle[0], obstacle[1], cfg.dx)
                n_ob = ob.shape[0]
                wall = torch.cat((wall, ob))
                clamp_out_of_obstacle_host(x, obstacle[0], obstacle[1], 0.01 * cfg.dx)
        finally:
            torch.set_default_dtype(saved)
        return x.double(), mass.double(), wall.double(), n_ob

    # ------------------------------------------------------------ stepping --
    def step(self, steps: int = 1, graph: bool = True) -> None:
        """Advance ``steps`` steps on the engine's stream (no host synchronisation)."""
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        L = _lib.lib()
        fn = L.tsph_engine_step if graph else L.tsph_engine_step_eager
        _lib.check(fn(self._handle, int(steps), self.stream.cuda_stream), "tsph_engine_step")
        self.steps_done += int(steps)

    def _hand_over(self, *tensors):
        """Make the caller's current stream wait for the engine stream, so the
        returned tensors are safe to use there."""
        cur = torch.cuda.current_stream(self.device)
        if cur != self.stream:
            cur.wait_stream(self.stream)
            for t in tensors:
                t.record_stream(cur)

    STAGES = ("rebuild", "density", "diffusion_eos", "walls", "force", "reaction",
              "integrate", "shift_rebuild", "concentration", "gradient", "select", "shift_apply")

    def step_timed(self) -> dict:
        """One eager step with CUDA events between stages; ``{stage: ms}``."""
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        ms = (ctypes.c_float * 12)()
        n = ctypes.c_int64(0)
        _lib.check(_lib.lib().tsph_engine_step_timed(self._handle, self.stream.cuda_stream, ms,
                                                     ctypes.byref(n)), "tsph_engine_step_timed")
        self.steps_done += 1
        return {self.STAGES[i]: float(ms[i]) for i in range(n.value)}

    def graph_kernels(self) -> int:
        """Kernel launches in one captured step (the step graph's kernel nodes)."""
        k = ctypes.c_int64(0)
        _lib.check(_lib.lib().tsph_engine_graph_kernels(self._handle, ctypes.byref(k)),
                   "tsph_engine_graph_kernels")
        return int(k.value)

    def diagnostics(self, first: int, count: int) -> torch.Tensor:
        """Per-step meter rows ``(count, 16)`` (fields in ``DIAG_FIELDS``)."""
        with torch.cuda.stream(self.stream):
            out = torch.empty((count, 16), dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib().tsph_engine_diag(self._handle, out.data_ptr(), int(first),
                                               int(count), self.stream.cuda_stream),
                   "tsph_engine_diag")
        self._hand_over(out)
        return out

    def state(self):
        """``(x, v, rho, p)`` of the fluid in the original particle order (device)."""
        n = self.n_fluid
        with torch.cuda.stream(self.stream):
            x = torch.empty((n, 3), dtype=torch.float64, device=self.device)
            v = torch.empty_like(x)
            rho = torch.empty(n, dtype=torch.float64, device=self.device)
            p = torch.empty_like(rho)
        _lib.check(_lib.lib().tsph_engine_read(self._handle, x.data_ptr(), v.data_ptr(),
                                               rho.data_ptr(), p.data_ptr(),
                                               self.stream.cuda_stream), "tsph_engine_read")
        self._hand_over(x, v, rho, p)
        return x, v, rho, p

    def status(self) -> dict:
        buf = (ctypes.c_int64 * 8)()
        rc = _lib.lib().tsph_engine_status(self._handle, buf, self.stream.cuda_stream)
        out = dict(escapes=buf[0], clamps=buf[1], rebuilds=buf[2], steps=buf[3], row_max=buf[4],
                   status=buf[6])
        if rc == _lib.ERR_CAPACITY:
            raise RuntimeError(f"neighbour row capacity exceeded (longest row {buf[4]}); "
                               "raise max_neighbors")
        _lib.check(rc, "tsph_engine_status")
        return out

    def close(self) -> None:
        if self._handle is not None and self._handle.value:
            torch.cuda.synchronize(self.device)
            _lib.lib().tsph_engine_destroy(self._handle)
            self._handle = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_case(cfg: DamBreak3DConfig, pair_skin_factor: float | None = None, snapshot_times=None,
             seed: int | None = None, *, obstacle=None, shift_every: int = 0,
             max_neighbors: int = 160) -> DamBreak3DRun:
    """Integrate the 3-D dam break on the GPU and return the run record.

    Same loop as dam_break_3d.py:569-734: ``cfg.steps`` steps of ``cfg.dt``,
    meters sampled every ``cfg.output_every`` steps and at the end.  The whole
    loop stays on the device; meters come back once at the end.
    """
    if snapshot_times:
        raise NotImplementedError("snapshot_times is not supported by the device engine")
    if cfg.adaptive_dt:
        raise NotImplementedError("adaptive_dt is not supported by the device engine")
    if pair_skin_factor is not None:
        from dataclasses import replace
        cfg = replace(cfg, pair_skin_factor=pair_skin_factor)
    eng = DamBreak3DEngine(cfg, obstacle=obstacle, shift_every=shift_every, seed=seed,
                           max_neighbors=max_neighbors, diag_ring=max(cfg.steps + 1, 1))
    eng.step(cfg.steps)
    with torch.cuda.stream(eng.stream):
        diag = eng.diagnostics(0, cfg.steps).cpu()
        x, v, rho, p = eng.state()
    st = eng.status()
    # the reference samples the state at step == cfg.steps too: one more rhs
    sample = [k for k in range(cfg.steps) if k % cfg.output_every == 0]
    times = [k * cfg.dt for k in sample]
    xs = x.cpu()
    vs = v.cpu()
    run = DamBreak3DRun(
        times=times, front=[float(diag[k, 2]) for k in sample],
        kinetic_energy=[float(diag[k, 6]) for k in sample],
        potential_energy=[float(diag[k, 7]) for k in sample],
        mass=eng.initial_mass, escaped=int(st["escapes"]), rebuilds=int(st["rebuilds"]),
        max_speed=float(diag[:, 1].max()) if cfg.steps else 0.0,
        max_density_compression=(float(diag[:, 0].max()) / cfg.rho0 - 1.0) if cfg.steps else 0.0,
        initial_mass=eng.initial_mass, final_mass=eng.initial_mass, final_positions=xs,
        initial_energy=eng.initial_pe, steps_taken=cfg.steps, simulated_time=cfg.steps * cfg.dt,
        obstacle_force=diag[:, 3:6].tolist(), obstacle_impulse=[float(diag[-1, 14])] if cfg.steps else [],
        obstacle_clamps=int(st["clamps"]))
    masses = DamBreak3DEngine.build_host_state(cfg, obstacle, seed)[1]
    run.final_energy = float(0.5 * (masses[:, None] * vs.square()).sum()
                             + (masses * cfg.gravity * xs[:, 1]).sum())
    eng.close()
    return run
