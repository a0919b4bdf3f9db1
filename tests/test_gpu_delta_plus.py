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
