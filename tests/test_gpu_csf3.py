"""3-D CSF drop-in (csf_fields3 / surface_tension_acceleration3, "mls") on the
GPU against the reference's own output (tests/golden/csf3.npz) and the
oracle.

Tolerances, relative to each field's largest magnitude: FP64 1e-11 (the
device sums rows in a fixed gather order and inverts M by its adjugate where
the reference scatters with index_add and solves by LU); FP32 2e-4 against
the reference's FP32 run (the curvature differentiates the normal, which
amplifies summation-order differences by ~R/dx).  Case 0 is the perfect
lattice ball, whose interior |grad c| is round-off: compared on the
acceleration only (1e-4), as the oracle is.
"""
import numpy as np
import pytest
import torch

from tests.test_oracle_golden import _csf3_case

pytestmark = pytest.mark.gpu


def _run(c):
    from tensorsph_b200.threed.csf3 import csf_fields3, surface_tension_acceleration3
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st = csf_fields3(t(c["pos"]), t(c["mass"]), c["h"], t(c["pairs"]), rho0=1000.0, box=c["box"],
                     volume=None if c["volume"] is None else t(c["volume"]))
    acc = surface_tension_acceleration3(st, t(c["rho"]), 0.0728)
    return st, acc


def test_csf3_fields_match_reference(golden, gpu):
    g = golden("csf3")
    for k in range(int(g["count"])):
        c = _csf3_case(g, k)
        st, acc = _run(c)
        f64 = c["pos"].dtype == np.float64
        ref = g[f"c{k}_acc"]
        got = acc.cpu().numpy()
        atol = (1e-4 if k == 0 else (1e-11 if f64 else 2e-4)) * np.abs(ref).max()
        assert np.abs(got - ref).max() <= atol, (k, np.abs(got - ref).max() / np.abs(ref).max())
        if k == 0:
            continue
        assert (st.valid.cpu().numpy() == g[f"c{k}_valid"]).all(), k
        tol = 1e-11 if f64 else 2e-4
        for name in ("color", "grad_c", "delta_s", "normal", "kappa"):
            r = g[f"c{k}_{name}"]
            d = np.abs(getattr(st, name).cpu().numpy() - r).max() / max(np.abs(r).max(), 1.0)
            assert d <= tol, (k, name, d)


def test_csf3_degenerate_stencils_fall_back(golden, gpu):
    """The stray particles of case 3 (an isolated particle and a close pair)
    have |det M| far below the median: not valid, kappa and force zero."""
    g = golden("csf3")
    c = _csf3_case(g, 3)
    st, acc = _run(c)
    valid = st.valid.cpu().numpy()
    assert not valid[-3:].any() and valid[:-3].all()
    assert (st.kappa.cpu().numpy()[-3:] == 0).all()
    assert (acc.cpu().numpy()[-3:] == 0).all()


def test_csf3_column_force_points_inward_and_vanishes_without_sigma(golden, gpu):
    """The periodic Rayleigh-Plateau column (case 4): with sigma = 0 the
    acceleration is zero, and on the interface shell the CSF force pulls
    toward the axis (the reference's own check, test_rayleigh_plateau.py)."""
    from tensorsph_b200.threed.csf3 import surface_tension_acceleration3
    g = golden("csf3")
    c = _csf3_case(g, 4)
    st, acc = _run(c)
    rho = torch.full((c["pos"].shape[0],), 1000.0, dtype=torch.float64, device="cuda")
    assert float(surface_tension_acceleration3(st, rho, 0.0).abs().max()) == 0.0
    shell = (st.surface_mask(0.3) & st.valid).cpu().numpy()
    box = c["box"]
    offset = c["pos"][:, :2] - 0.5 * box[:2]
    radial = offset[shell] / np.linalg.norm(offset[shell], axis=1)[:, None]
    a = acc.cpu().numpy()[shell]
    cos = (a[:, :2] * radial).sum(axis=1) / np.maximum(np.linalg.norm(a, axis=1), 1e-30)
    assert cos.mean() < -0.8


def test_csf3_matches_oracle_on_a_larger_jittered_ball(gpu):
    """A 6,000-particle jittered ball centred on a corner of a periodic box,
    so that its pairs and sums cross the wrap on every axis: device against
    the oracle (FP64, 1e-11)."""
    from oracle import csf3 as oc
    from oracle.neighbors import periodic_pairs
    rng = np.random.default_rng(5)
    dx = 1e-3
    ax = np.arange(-12, 13) * dx
    pts = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    pts = pts[np.linalg.norm(pts, axis=1) <= 11.3 * dx] + rng.uniform(-0.1, 0.1, (1, 3)) * dx
    pts = pts + 0.1 * dx * rng.standard_normal(pts.shape)
    box = np.array([0.04, 0.04, 0.04])
    pos = np.mod(pts, box)
    mass = np.full(pos.shape[0], 1000.0 * dx ** 3)
    rho = 1000.0 * (1.0 + 0.002 * rng.standard_normal(pos.shape[0]))
    h = 1.3 * dx
    pairs = periodic_pairs(pos, box, 2.0 * h)
    ref = oc.csf_fields3(pos, mass, h, pairs, rho0=1000.0, box=box)
    ref_acc = oc.surface_tension_acceleration3(ref, rho, 0.0728)
    c = dict(pos=pos, mass=mass, rho=rho, pairs=pairs, h=h, box=box, volume=None)
    st, acc = _run(c)
    assert (st.valid.cpu().numpy() == ref["valid"]).all()
    for name in ("color", "grad_c", "delta_s", "normal", "kappa"):
        r = ref[name]
        d = np.abs(getattr(st, name).cpu().numpy() - r).max() / max(np.abs(r).max(), 1.0)
        assert d <= 1e-11, (name, d)
    assert np.abs(acc.cpu().numpy() - ref_acc).max() <= 1e-11 * np.abs(ref_acc).max()


def test_csf3_axisym_matches_reference(golden, gpu):
    """csf_fields3(curvature="axisym") on 4h lists (a jittered ball in FP64
    and FP32, the periodic liquid column in FP64) against the reference's own
    output (tests/golden/csf3axi.npz): the curvature of the surface particles
    (delta_s > 1e-3 max) within 1e-9 (FP64) / 1e-3 (FP32) of its largest
    value, and the acceleration the same."""
    from tensorsph_b200.threed.csf3 import csf_fields3, surface_tension_acceleration3
    g = golden("csf3axi")
    for k in range(int(g["count"])):
        pos = g[f"c{k}_pos"]
        box = g[f"c{k}_box"]
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        st = csf_fields3(dev(pos), dev(g[f"c{k}_mass"]), float(g[f"c{k}_h"]), dev(g[f"c{k}_pairs"]),
                         rho0=1000.0, box=None if not box.any() else box.tolist(), curvature="axisym")
        tol = 1e-9 if pos.dtype == np.float64 else 1e-3
        live = g[f"c{k}_delta_s"] > 1e-3 * g[f"c{k}_delta_s"].max()
        r = g[f"c{k}_kappa"][live]
        got = st.kappa.cpu().numpy()[live]
        assert np.abs(got - r).max() <= tol * np.abs(r).max(), k
        acc = surface_tension_acceleration3(st, dev(g[f"c{k}_rho"]), 0.0728).cpu().numpy()
        ra = g[f"c{k}_acc"]
        assert np.abs(acc - ra).max() <= tol * np.abs(ra).max(), k
