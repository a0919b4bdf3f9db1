"""The dimension-generic delta-plus oracle in 3-D (CPU).

In 2-D it is pinned to the reference's fixtures (test_oracle_golden.py); in
3-D there is no reference step, so these checks state what the 3-D
statements must give by symmetry: free flight of a lone particle, no force
and no shift on the interior of a uniform lattice, and the 3-D Wendland
normalisation (int W dV = 1 over the 2h ball).
"""
import math

import numpy as np

from oracle import delta_plus as odp

KW = dict(dx=0.01, sound_speed=20.0, reference_speed=0.5, dt=1e-4, gravity=0.0, viscosity=1e-6,
          diffusion=0.1, alpha=0.02)


def test_lone_particle_flies_free():
    pos = np.array([[0.1, 0.2, 0.3]])
    vel = np.array([[0.5, -0.25, 0.125]])
    out = odp.delta_plus_step(pos, vel, np.array([1003.0]), np.array([1e-3]), **KW)
    assert np.array_equal(out["position"], pos + KW["dt"] * vel)
    assert np.array_equal(out["density"], np.array([1003.0]))
    assert not out["shift"].any()


def test_uniform_lattice_interior_is_at_rest():
    ax = (np.arange(11) + 0.5) * 0.01
    pos = np.stack([a.ravel() for a in np.meshgrid(ax, ax, ax, indexing="ij")], 1)
    rho = np.full(pos.shape[0], 1000.0)
    out = odp.delta_plus_step(pos, np.zeros_like(pos), rho, rho * 1e-6, **KW)
    mid = np.all(np.abs(pos - 0.055) < 0.011, axis=1)      # the 27 central particles
    assert mid.sum() == 27
    assert np.abs(out["acceleration"][mid]).max() < 1e-9
    assert np.abs(out["shift"][mid]).max() < 1e-18
    assert np.abs(out["density"][mid] - 1000.0).max() < 1e-9


def test_wendland_3d_normalisation():
    h = 0.02
    r = np.linspace(0.0, 2 * h, 200001)
    w = odp.wendland(r, h, 3)
    integral = np.trapezoid(4 * math.pi * r * r * w, r)
    assert abs(integral - 1.0) < 1e-8
