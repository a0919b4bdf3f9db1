"""Periodic shear-wave decay on the device against the reference's own run
(tests/golden/shear.npz: threed/solver.py run_shear_wave, n = 12, 40 steps).

FP64: the sampled mode amplitudes and energies agree to 1e-10 relative and
the pair count and rebuild count exactly.  FP32 (compensated pair sums
against the reference's plain FP32 torch sums): amplitudes to 1e-5 relative.
The single-mode variant is checked for the FP32/FP64 agreement of its decay
rate and density field.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_shear_wave_matches_reference(golden, gpu):
    from tensorsph_b200.threed.shear import run_shear_wave
    g = golden("shear")
    for k, dtype in ((0, torch.float64), (1, torch.float32)):
        r = run_shear_wave(n=12, steps=40, sample_every=10, dtype=dtype)
        amp = np.asarray(r.amplitudes)
        ref = g[f"c{k}_amplitudes"]
        assert np.allclose(r.times, g[f"c{k}_times"], rtol=0, atol=1e-15)
        tol = 1e-10 if dtype == torch.float64 else 1e-5
        assert np.abs(amp - ref).max() <= tol * np.abs(ref).max(), (k, amp, ref)
        ke = np.asarray([d["kinetic_energy"] for d in r.diagnostics])
        assert np.abs(ke - g[f"c{k}_kinetic"]).max() <= tol * 10 * np.abs(g[f"c{k}_kinetic"]).max()
        if dtype == torch.float64:
            te = np.asarray([d["total_energy"] for d in r.diagnostics])
            assert np.abs(te - g[f"c{k}_total"]).max() <= 1e-9 * np.abs(g[f"c{k}_total"]).max()
            assert r.pairs_last == int(g[f"c{k}_pairs_last"])
            assert r.pair_rebuilds == int(g[f"c{k}_rebuilds"])
            assert r.fit_rate == pytest.approx(float(g[f"c{k}_fit_rate"]), rel=1e-8)


def test_single_mode_decay_fp32_matches_fp64(gpu):
    from tensorsph_b200.threed.shear import run_shear_decay
    kw = dict(n=24, steps=300, sample_every=30, amplitude=1e-3, nu=1e-2, sound_speed=1.0)
    a = run_shear_decay(dtype=torch.float32, **kw)      # FP32 pairs on an FP64 state
    b = run_shear_decay(dtype=torch.float64, **kw)
    assert abs(a.fit_rate - b.fit_rate) <= 1e-3 * abs(b.fit_rate)
    drho = (a.final_density.double() - b.final_density).abs().max().item()
    assert drho / 1000.0 < 1e-5
    # the jittered lattice starts with a small momentum; its drift stays at
    # round-off of the momentum the flow carries
    p0 = np.asarray(b.diagnostics[0]["momentum"])
    p1 = np.asarray(b.diagnostics[-1]["momentum"])
    assert np.abs(p1 - p0).max() <= 1e-10 * b.momentum_scale
