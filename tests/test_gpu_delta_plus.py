"""The 2-D delta-plus step on the GPU against the reference's own outputs
(tests/golden/delta_plus.npz) and against the physical statements the
reference's tests check: free flight, the eq. (5) shift of an interior
particle as a direct sum, linear scaling of the shift with dt, and a
diffusion term that leaves an affine density profile alone.

FP64 fields agree to 1e-12 relative to the field's largest value; FP32 ones
to 5e-6 (the interface band is a set of thresholds on lambda, identical here).
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KW = dict(dx=0.01, sound_speed=20.0, reference_speed=0.5, dt=1e-4, gravity=9.81, viscosity=1e-6,
          diffusion=0.1, alpha=0.02)


def test_delta_plus_matches_reference(golden, gpu):
    from tensorsph_b200.delta_plus import delta_plus_step
    g = golden("delta_plus")
    for k in range(int(g["count"])):
        t = {n: torch.from_numpy(g[f"c{k}_{n}"]).cuda() for n in ("pos", "vel", "rho", "mass")}
        wall = torch.from_numpy(g[f"c{k}_wall"]).cuda() if f"c{k}_wall" in g else None
        wn = torch.from_numpy(g[f"c{k}_wall_normal"]).cuda() if wall is not None else None
        out = delta_plus_step(t["pos"], t["vel"], t["rho"], t["mass"], wall=wall, wall_normal=wn,
                              wall_velocity=None if wall is None else torch.zeros_like(wall), **KW)
        tol = 1e-12 if t["pos"].dtype == torch.float64 else 5e-6
        for key in ("position", "velocity", "density", "acceleration", "wall_reaction", "shift"):
            ref = g[f"c{k}_out_{key}"]
            if not ref.size:
                continue
            got = getattr(out, key).cpu().numpy()
            assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (k, key)


def _lattice(n=15, dx=0.01):
    ax = (torch.arange(n, dtype=torch.float64) + 0.5) * dx
    pos = torch.cartesian_prod(ax, ax).cuda()
    rho = torch.full((pos.shape[0],), 1000.0, dtype=torch.float64, device="cuda")
    return pos, torch.zeros_like(pos), rho, rho * dx * dx


def test_free_flight_and_direct_shift(gpu):
    from tensorsph_b200.delta_plus import delta_plus_step
    opts = dict(dx=0.01, sound_speed=20.0, reference_speed=0.5, dt=1e-4, gravity=0.0)
    pos, vel, rho, mass = _lattice(2)
    p1, v1, r1, m1 = pos[:1], vel[:1] + 0.25, rho[:1] + 3.0, mass[:1]
    st = delta_plus_step(p1, v1, r1, m1, **opts)
    assert torch.allclose(st.position, p1 + v1 * opts["dt"], atol=1e-15, rtol=0)
    assert torch.equal(st.density, r1) and torch.count_nonzero(st.shift) == 0
    # eq. (5) shift of an interior particle as a direct sum over its support
    pos, vel, rho, mass = _lattice()
    mid = 7 * 15 + 7
    pos[mid, 0] += 0.23 * 0.01
    st = delta_plus_step(pos, vel, rho, mass, **opts)
    h = 0.02
    x = pos[mid] - pos
    q = x.norm(dim=1) / h
    t = (1 - q / 2).clamp_min(0)
    sigma = 7 / (4 * math.pi * h * h)
    wgt = sigma * t ** 4 * (2 * q + 1)
    w_dx = sigma * (1 - 0.25) ** 4 * 2
    grad = (-5 * sigma / h ** 2 * t ** 3)[:, None] * x
    raw = ((1 + 0.2 * (wgt / w_dx) ** 4) * mass / (rho + rho[mid]))[:, None] * grad
    expect = -4 * h * opts["dt"] * opts["reference_speed"] * raw.sum(0)
    assert torch.allclose(st.shift[mid], expect, rtol=2e-12, atol=1e-15)
    # the shift is linear in dt
    half = delta_plus_step(pos, vel, rho, mass, **dict(opts, dt=opts["dt"] / 2))
    assert torch.allclose(half.shift * 2, st.shift, rtol=1e-12, atol=1e-14)


def test_diffusion_keeps_affine_profile(gpu):
    from tensorsph_b200.delta_plus import delta_plus_step
    opts = dict(dx=0.01, sound_speed=20.0, reference_speed=0.0, dt=1e-4, gravity=0.0)
    pos, vel, rho, _ = _lattice()
    r = rho + 3 * (pos[:, 1] - 0.1)
    m = r * 1e-4
    a = delta_plus_step(pos, vel, r, m, diffusion=0.1, **opts)
    b = delta_plus_step(pos, vel, r, m, diffusion=0.0, **opts)
    interior = ((pos - 0.075).abs() < 0.04).all(dim=1)
    assert torch.allclose(a.density[interior], b.density[interior], rtol=0, atol=1e-9)
    noisy = rho + 0.15 * (-1.0) ** torch.arange(len(pos), device="cuda")
    c = delta_plus_step(pos, vel, noisy, noisy * 1e-4, diffusion=0.1, **opts)
    d = delta_plus_step(pos, vel, noisy, noisy * 1e-4, diffusion=0.0, **opts)
    dev_c = (c.density[interior] - 1000.0).abs().mean()
    dev_d = (d.density[interior] - 1000.0).abs().mean()
    assert dev_c < dev_d


def walled_corner_3d(dtype=np.float64, seed=3, dx=0.01):
    """A jittered 7 x 5 x 6 fluid block on four floor layers of stations
    (normal +y) beside four layers of a side wall (normal +x): a free
    surface, a wall and a wall corner in 3-D."""
    rng = np.random.default_rng(seed)
    ax = lambda k: (np.arange(k) + 0.5) * dx  # noqa: E731
    X, Y, Z = np.meshgrid(ax(7), ax(5), ax(6), indexing="ij")
    pos = np.stack((X.ravel(), Y.ravel(), Z.ravel()), 1)
    pos = pos + rng.uniform(-0.08, 0.08, pos.shape) * dx
    wx = (np.arange(-4, 9) + 0.5) * dx
    wz = (np.arange(-2, 8) + 0.5) * dx
    floor = np.stack([a.ravel() for a in np.meshgrid(wx, (np.arange(-4, 0) + 0.5) * dx, wz, indexing="ij")], 1)
    side = np.stack([a.ravel() for a in np.meshgrid((np.arange(-4, 0) + 0.5) * dx, ax(8), wz, indexing="ij")], 1)
    wall = np.concatenate((floor, side))
    normal = np.zeros_like(wall)
    normal[: floor.shape[0], 1] = 1.0
    normal[floor.shape[0]:, 0] = 1.0
    rho = 1000.0 * (1.0 + 0.002 * rng.standard_normal(pos.shape[0]))
    vel = 0.05 * rng.standard_normal(pos.shape)
    mass = 1000.0 * dx ** 3 * np.ones(pos.shape[0])
    return tuple(a.astype(dtype) for a in (pos, vel, rho, mass, wall, normal))


KW3 = dict(dx=0.01, sound_speed=20.0, reference_speed=0.5, dt=1e-4, gravity=9.81, viscosity=1e-6,
           diffusion=0.1, alpha=0.02)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 5e-5)])
def test_delta_plus_3d_matches_oracle(dtype, tol, gpu):
    """delta_plus_step3 against the dimension-generic oracle (the 2-D step's
    statements for D = 3, pinned in 2-D to the reference's fixtures) on a
    walled corner: every output field within tol of the field's largest
    value, in the input dtype (FP32 against the oracle in FP32)."""
    from oracle import delta_plus as odp
    from tensorsph_b200.delta_plus import delta_plus_step3
    pos, vel, rho, mass, wall, normal = walled_corner_3d(dtype)
    ref = odp.delta_plus_step(pos, vel, rho, mass, wall=wall, wall_velocity=np.zeros_like(wall),
                              wall_normal=normal, **KW3)
    t = [torch.from_numpy(a).cuda() for a in (pos, vel, rho, mass, wall, normal)]
    out = delta_plus_step3(t[0], t[1], t[2], t[3], wall=t[4], wall_velocity=torch.zeros_like(t[4]),
                           wall_normal=t[5], **KW3)
    assert np.abs(ref["shift"]).max() > 1e-9
    for key in ("position", "velocity", "density", "acceleration", "wall_reaction", "shift"):
        want = ref[key]
        got = getattr(out, key).cpu().numpy()
        assert np.abs(got - want).max() <= tol * np.abs(want).max(), (key, np.abs(got - want).max())


def test_delta_plus_3d_rejects_2d_input(gpu):
    from tensorsph_b200.delta_plus import delta_plus_step, delta_plus_step3
    pos, vel, rho, mass, wall, normal = walled_corner_3d()
    t = [torch.from_numpy(a).cuda() for a in (pos, vel, rho, mass)]
    with pytest.raises(ValueError):
        delta_plus_step(t[0], t[1], t[2], t[3], **KW3)        # the reference's 2-D contract
    with pytest.raises(ValueError):
        delta_plus_step3(t[0][:, :2].contiguous(), t[1][:, :2].contiguous(), t[2], t[3], **KW3)


def test_delta_plus_dam_break_3d_runs(gpu):
    """The 3-D delta-plus dam break with the obstacle on a coarse lattice:
    the first step against the oracle, then 12 steps from the hydrostatic
    start stay finite with a bounded density deviation."""
    from oracle import delta_plus as odp
    from tensorsph_b200.engine import obstacle_case
    from tensorsph_b200.threed.delta_plus3 import delta_plus_case_3d, run_delta_plus_3d
    cfg, obstacle = obstacle_case(dx=0.04)
    host = delta_plus_case_3d(cfg, obstacle, torch.float64)
    one = run_delta_plus_3d(cfg, 1, obstacle=obstacle, host_state=host, device=gpu)
    pos, rho, mass, wall, normal, n_ob = (t.numpy() if torch.is_tensor(t) else t for t in host)
    h = 2.0 * cfg.dx
    ref = odp.delta_plus_step(pos, np.zeros_like(pos), rho, mass, dx=cfg.dx, sound_speed=cfg.sound_speed,
                              reference_speed=math.sqrt(2 * cfg.gravity * cfg.column_height),
                              dt=cfg.max_courant * h / cfg.sound_speed, rho0=cfg.rho0, gravity=cfg.gravity,
                              viscosity=cfg.viscosity, wall=wall, wall_velocity=np.zeros_like(wall),
                              wall_normal=normal)
    assert np.abs(one.final_positions.cpu().numpy() - ref["position"]).max() < 1e-9 * cfg.dx
    assert np.abs(one.final_density.cpu().numpy() - ref["density"]).max() < 1e-9 * cfg.rho0
    run = run_delta_plus_3d(cfg, 12, obstacle=obstacle, host_state=host, device=gpu)
    assert torch.isfinite(run.final_positions).all()
    assert max(run.density_deviation) < 0.02
    assert n_ob > 0 and len(run.obstacle_force) == 12
