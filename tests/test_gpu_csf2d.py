"""2-D CSF drop-in (csf_fields / surface_tension_acceleration with the
"mls", "fit_quadratic" and "fit_circle" curvatures, "legacy" and "local_range" delta_s,
normal smoothing off, curvature from a smoothed colour) on the GPU against
the reference's own outputs (tests/golden/csf2d.npz, csf.npz).

Tolerances, relative to each field's largest magnitude: FP64 1e-11 on the
colour, its gradient and delta_s, 1e-8 on the normal, the curvature and the
acceleration (the Shepard passes average in interior normals whose
directions are those of round-off-sized gradients, so the smoothed surface
normal carries the summation order at ~1e-10); FP32 1e-4 and 1e-3
(differentiating the colour twice amplifies the FP32 summation differences;
the reference's own FP32 run is further from its FP64 run).
Normals and curvatures are compared where delta_s > 0: interior normals are
round-off directions.
"""
import ast

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _compare(st, acc, g, k, f64, directions=True):
    live = g[f"c{k}_delta_s"] > 0
    tol_a = 1e-11 if f64 else 1e-4
    for name in ("color", "grad_c", "delta_s"):
        r = g[f"c{k}_{name}"]
        d = np.abs(getattr(st, name).cpu().numpy() - r).max() / max(np.abs(r).max(), 1.0)
        assert d <= tol_a, (k, name, d)
    if not directions:
        return
    tol_b = 1e-8 if f64 else 1e-3
    for name in ("normal", "kappa"):
        r = g[f"c{k}_{name}"][live]
        d = np.abs(getattr(st, name).cpu().numpy()[live] - r).max() / np.abs(r).max()
        assert d <= tol_b, (k, name, d)
    if acc is not None:
        r = g[f"c{k}_acc"]
        d = np.abs(acc.cpu().numpy() - r).max() / np.abs(r).max()
        assert d <= tol_b, (k, "acc", d)


def test_csf2d_variants_match_reference(golden, gpu):
    from tensorsph_b200 import csf_consistent as cc
    g = golden("csf2d")
    for k in range(int(g["count"])):
        o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
        pos, mass, rho, pairs, h = (g[f"c{k}_pos"], g[f"c{k}_mass"], g[f"c{k}_rho"], g[f"c{k}_pairs"],
                                    float(g[f"c{k}_h"]))
        if int(g[f"c{k}_direct"]):
            st = cc.csf_fields(_t(pos), _t(mass), _t(pairs), h, 1000.0, **o)
            acc = None
        else:
            acc, st = cc.surface_tension_acceleration(_t(pos), _t(rho), _t(mass), _t(pairs), h, 0.0728,
                                                      rho0=1000.0, **o)
        _compare(st, acc, g, k, pos.dtype == np.float64)


def test_csf2d_default_fit_matches_reference_fixture(golden, gpu):
    """The fixtures of the droplet case's CSF (fit_quadratic, legacy) through
    the standalone drop-in.  On the FP32 lattice drops the interior colour
    gradients are FP32 round-off above the 1e-12 normal threshold, so the
    interior normals are arbitrary unit vectors that the Shepard passes mix
    into the surface normals (in the reference as here): those cases compare
    the colour, its gradient and delta_s only."""
    from oracle.neighbors import cell_linked_pairs
    from tensorsph_b200 import csf_consistent as cc
    g = golden("csf")
    for k in range(int(g["count"])):
        pos = g[f"c{k}_pos"]
        h = float(g[f"c{k}_h"])
        pairs = cell_linked_pairs(pos, 2.0 * h)
        acc, st = cc.surface_tension_acceleration(_t(pos), _t(g[f"c{k}_rho"]), _t(g[f"c{k}_mass"]), _t(pairs), h,
                                                  0.0728, rho0=1000.0, curvature_scheme="fit_quadratic")
        f64 = pos.dtype == np.float64
        _compare(st, acc, g, k, f64, directions=f64)


def test_csf2d_options_and_errors(gpu):
    from tensorsph_b200 import csf_consistent as cc
    pos = torch.rand((50, 2), dtype=torch.float64, device="cuda") * 0.01
    mass = torch.full((50,), 1e-3, dtype=torch.float64, device="cuda")
    pairs = torch.zeros((0, 2), dtype=torch.int64, device="cuda")
    a, st = cc.surface_tension_acceleration(pos, mass * 1e6, mass, pairs, 0.002, 0.0)
    assert st is None and float(a.abs().max()) == 0.0
    with pytest.raises(ValueError):
        cc.csf_fields(pos, mass, pairs, 0.002, 1000.0, curvature_scheme="fit_ellipse")
    with pytest.raises(ValueError):
        cc.csf_fields(pos, mass, pairs, 0.002, 1000.0, delta_normalization="other")
    with pytest.raises(ValueError):
        cc.surface_tension_acceleration(pos, mass * 1e6, mass, pairs, 0.002, 0.07, wall=pos, contact_angle=1.0,
                                        contact_angle_model="hoffman")
    with pytest.raises(ValueError):
        cc.surface_tension_acceleration(pos, mass * 1e6, mass, pairs, 0.002, 0.07, contact_angle=1.0,
                                        wall=pos[:0], contact_angle_model="young")


def test_nearest_wall_and_boundary_match_reference(golden, gpu):
    """nearest_wall (with a particle sitting on a wall particle: the mean
    direction of the others) and apply_contact_angle_boundary at 30 and 120
    degrees against the reference (tests/golden/contact.npz), FP64."""
    from tensorsph_b200 import csf_consistent as cc
    g = golden("contact")
    wall, h = _t(g["wall"]), float(g["h"])
    d, nrm = cc.nearest_wall(_t(g["nw_pos"]), wall)
    assert np.abs(d.cpu().numpy() - g["nw_dist"]).max() <= 1e-15
    assert np.abs(nrm.cpu().numpy() - g["nw_normal"]).max() <= 1e-12
    pos = _t(g["nw_pos"][:-1])
    for k in range(2):
        out = cc.apply_contact_angle_boundary(_t(g["bc_grad"]), pos, wall, h, float(g[f"bc{k}_theta"]))
        ref = g[f"bc{k}_out"]
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max(), k


def test_contact_angle_csf_matches_reference(golden, gpu):
    """The CSF with the "rotate" boundary (mls and fit_quadratic curvature,
    and through csf_fields with a smoothed-colour curvature) and with the
    "young" and "brackbill" tractions on a sessile half-drop, FP64 and FP32,
    against the reference.  The traction is a small part of the force (0.2-0.4 %
    of the largest acceleration), so it is also compared on its own: this
    path's acceleration minus its acceleration without the wall, against the
    reference's acceleration minus the oracle's without the wall, to 1e-8
    (FP64) / 1e-3 (FP32) of the traction's largest value."""
    import ast

    from oracle import csf as ocsf
    from tensorsph_b200 import csf_consistent as cc
    g = golden("contact")
    h = float(g["h"])
    for k in range(int(g["count"])):
        o = dict(ast.literal_eval(str(g[f"c{k}_opts"])))
        pos, mass, rho, pairs = g[f"c{k}_pos"], g[f"c{k}_mass"], g[f"c{k}_rho"], g[f"c{k}_pairs"]
        wall = _t(g["wall"].astype(pos.dtype))
        f64 = pos.dtype == np.float64
        if int(g[f"c{k}_direct"]):
            st = cc.csf_fields(_t(pos), _t(mass), _t(pairs), h, 1000.0, wall=wall, **o)
            acc = None
        else:
            acc, st = cc.surface_tension_acceleration(_t(pos), _t(rho), _t(mass), _t(pairs), h, 0.0728,
                                                      rho0=1000.0, wall=wall, **o)
        _compare(st, acc, g, k, f64)
        if acc is not None and o["contact_angle_model"] != "rotate":
            bare, _ = cc.surface_tension_acceleration(_t(pos), _t(rho), _t(mass), _t(pairs), h, 0.0728,
                                                      rho0=1000.0, curvature_scheme=o["curvature_scheme"])
            ref_bare, _ = ocsf.surface_tension_acceleration(pos, rho, mass, h, 0.0728, 1000.0, pairs=pairs,
                                                            curvature_scheme=o["curvature_scheme"])
            mine = (acc - bare).cpu().numpy()
            ref = g[f"c{k}_acc"] - ref_bare
            assert np.abs(ref).max() > 0
            assert np.abs(mine - ref).max() <= (1e-8 if f64 else 1e-3) * np.abs(ref).max(), k


def test_contact_angle_boundary_properties(gpu):
    """The reference's own checks of the boundary (tests/test_contact_angle.py):
    no wall leaves the gradient unchanged, particles beyond the reach are
    untouched, |grad c| is kept, 90 degrees at the wall gives a normal along
    the wall."""
    import math

    from tensorsph_b200 import csf_consistent as cc
    grad = torch.tensor([[1.0, 0.0], [0.0, 1.0]], dtype=torch.float32, device="cuda")
    pos = torch.tensor([[0.1, 0.1], [0.2, 0.2]], dtype=torch.float32, device="cuda")
    empty = torch.empty((0, 2), dtype=torch.float32, device="cuda")
    assert torch.equal(cc.apply_contact_angle_boundary(grad, pos, empty, 0.1, math.pi / 4), grad)
    far_wall = torch.tensor([[0.0, -0.05], [0.1, -0.05]], dtype=torch.float32, device="cuda")
    far = torch.tensor([[0.5, 0.5]], dtype=torch.float32, device="cuda")
    g1 = torch.tensor([[1.0, 0.5]], dtype=torch.float32, device="cuda")
    assert torch.equal(cc.apply_contact_angle_boundary(g1, far, far_wall, 0.065, math.pi / 4), g1)
    wx = torch.arange(-8, 9, dtype=torch.float64, device="cuda") * 0.05
    wall = torch.stack((wx, torch.full_like(wx, -0.025)), -1)
    near = torch.tensor([[0.1, 0.02], [0.2, 0.03], [0.3, 0.08], [0.15, 0.5]], dtype=torch.float64, device="cuda")
    gn = torch.tensor([[0.5, 0.5], [0.3, 0.7], [0.1, 0.9], [0.8, 0.2]], dtype=torch.float64, device="cuda")
    for theta in (math.pi / 6, math.pi / 3, math.pi / 2, 2 * math.pi / 3):
        out = cc.apply_contact_angle_boundary(gn, near, wall, 0.065, theta)
        assert torch.allclose(out.norm(dim=1), gn.norm(dim=1), rtol=1e-12)
        assert torch.equal(out[3], gn[3])          # 0.5 m above the wall: beyond 2h
    # on the wall line (blend 1) at 90 degrees the normal lies along the wall
    on = torch.tensor([[0.0, -0.025 + 1e-9]], dtype=torch.float64, device="cuda")
    out = cc.apply_contact_angle_boundary(torch.tensor([[0.3, -0.4]], dtype=torch.float64, device="cuda"), on,
                                          wall, 0.065, math.pi / 2)
    assert abs(float(out[0, 1])) < 1e-6 * float(out.norm())
