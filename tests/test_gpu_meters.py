"""Device conservation meters and pair-list density against the reference's
own outputs (tests/golden/meters.npz).

The device sums are FP64; the reference sums in the input dtype, so FP32
fixtures agree to the FP32 summation error (2e-6 relative; the internal
energy, quadratic in rho - rho0, to 5e-3 relative) and FP64 ones to 1e-12.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_conservation_diagnostics_match_reference(golden, gpu):
    from tensorsph_b200.threed import conservation as cons
    g = golden("meters")
    for k in range(int(g["count"])):
        if int(g[f"c{k}_dim"]) != 3:
            continue
        pos, vel, mass, rho = (torch.from_numpy(g[f"c{k}_{n}"]).cuda() for n in ("pos", "vel", "mass", "rho"))
        box = float(g[f"c{k}_box"])
        row = cons.diagnostics(pos, vel, mass, rho, rho0=1000.0, sound_speed=20.0, gamma=7.0,
                               periodic_box=None if box < 0 else box)
        fp32 = pos.dtype == torch.float32
        tol = 2e-6 if fp32 else 1e-12
        for key in ("mass", "kinetic_energy", "momentum", "angular_momentum", "centre_of_mass"):
            ref = np.asarray(g[f"c{k}_ledger_{key}"])
            assert np.abs(np.asarray(row[key]) - ref).max() <= tol * max(np.abs(ref).max(), 1.0), (k, key)
        ie = float(g[f"c{k}_ledger_internal_energy"])
        assert abs(row["internal_energy"] - ie) <= (5e-3 if fp32 else 1e-9) * abs(ie)
        e = cons.internal_energy(rho, 1000.0, 20.0, 7.0).cpu().numpy()
        assert np.abs(e - g[f"c{k}_e"]).max() <= (2e-2 if fp32 else 1e-9) * np.abs(g[f"c{k}_e"]).max()
        assert cons.mass_total(mass) == pytest.approx(float(g[f"c{k}_ledger_mass"]), rel=tol)
        d = cons.relative_drift([1.0, 1.5, 0.9], scale=2.0)
        assert d["delta"] == pytest.approx(-0.1) and d["relative_drift"] == pytest.approx(-0.05)


def test_density_from_neighbor_pairs_matches_reference(golden, gpu):
    from tensorsph_b200.droplet_impact import density_from_neighbor_pairs
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    g = golden("meters")
    for k in range(int(g["count"])):
        pos = torch.from_numpy(g[f"c{k}_pos"]).cuda()
        mass = torch.from_numpy(g[f"c{k}_mass"]).cuda()
        pairs = cell_linked_pairs(pos, 0.06)
        got = density_from_neighbor_pairs(pos, mass, 0.03, pairs).cpu().numpy()
        ref = g[f"c{k}_rho_pairs"]
        tol = 2e-6 if pos.dtype == torch.float32 else 1e-12
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), k
        got2 = density_from_neighbor_pairs(pos, mass, 0.03).cpu().numpy()
        assert np.abs(got2 - ref).max() <= tol * np.abs(ref).max(), k
    with pytest.raises(ValueError):
        density_from_neighbor_pairs(pos, mass[:-1], 0.03)
    with pytest.raises(TypeError):
        density_from_neighbor_pairs(pos.long(), mass, 0.03)
