"""``run_hydrostatic`` (threed/solver.py:353-484) on the device against the
reference's own runs (tests/golden/hydrostatic.npz, written by running the
reference): a lidded column and an open one with psi-form density diffusion.
FP64 throughout; the sampled bottom pressure, centre of mass and the profile
(Eulerian and lattice rows, the depth integral, odd-even amplitude, binning
diagnostic) within 1e-9 relative."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    dict(nx=6, ny=5, nz=7, steps=30, sample_every=5, settle_fraction=0.5),
    dict(nx=5, ny=5, nz=6, steps=24, sample_every=4, settle_fraction=0.5, lid=False,
         density_diffusion=0.1, wall_model="adami"),
]


def _close(got, want, rel=1e-9):
    got, want = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape
    scale = max(float(np.abs(want).max()), 1e-300) if want.size else 1.0
    assert float(np.abs(got - want).max()) <= rel * scale, (got, want)


@pytest.mark.parametrize("k", range(len(CASES)))
def test_run_hydrostatic_follows_reference(k, golden, gpu):
    import torch
    from tensorsph_b200.threed import run_hydrostatic
    g = golden("hydrostatic")
    r = run_hydrostatic(dtype=torch.float64, device=gpu, **CASES[k])
    assert [r.steps, r.fluid_particles, r.wall_particles] == g[f"c{k}_counts"].tolist()
    _close(r.times, g[f"c{k}_times"], 1e-12)
    _close(r.bottom_pressure, g[f"c{k}_bottom"])
    _close(r.centre_of_mass_z, g[f"c{k}_com"], 1e-12)
    prof = r.profile
    _close([row["p_measured"] for row in prof["rows"]], g[f"c{k}_rows_p"])
    _close([row["rho_measured"] for row in prof["rows"]], g[f"c{k}_rows_rho"], 1e-12)
    _close([row["p_measured"] for row in prof["rows_by_lattice"]], g[f"c{k}_lat_p"])
    _close([row["z"] for row in prof["rows_by_lattice"]], g[f"c{k}_lat_z"], 1e-12)
    for key in ("integral_p_measured", "odd_even_amplitude_over_scale", "max_rel_error_core_lattice"):
        want = float(g[f"c{k}_{key}"])
        got = prof[key]
        if math.isnan(want):
            assert got is None
        else:
            assert got == pytest.approx(want, rel=1e-8, abs=1e-12), key
    assert prof["wall_displacement"] == float(g[f"c{k}_wall_displacement"])
    b = prof["binning"]
    _close([b["mean_offset_over_dx"], b["rms_offset_over_dx"], b["misplaced_fraction"]], g[f"c{k}_binning"], 1e-9)
    assert r.diagnostics[0]["kinetic_energy"] == pytest.approx(float(g[f"c{k}_kinetic"]), rel=1e-12)
