"""Shared check of a device run record against a reference run fixture."""
import numpy as np


def assert_follows(run, g, front_tol):
    """Engine trajectory against the reference's FP64 run: errors measured
    against what changed over the run (energies, positions), the front in
    metres.  The engine's FP32 pair sums give ~1e-5 relative acceleration
    errors, integrated over the run."""
    assert run.steps_taken == int(g["steps"]) and run.escaped == int(g["escaped"])
    assert np.allclose(run.times, g["times"], rtol=0, atol=1e-15)
    pe, ke = np.asarray(run.potential_energy), np.asarray(run.kinetic_energy)
    err = {
        "front": float(np.abs(np.asarray(run.front) - g["front"]).max()),
        "pe_vs_change": float(np.abs((pe - pe[0]) - (g["potential"] - g["potential"][0])).max()
                              / np.abs(g["potential"] - g["potential"][0]).max()),
        "ke": float(np.abs(ke - g["kinetic"]).max() / g["kinetic"].max()),
    }
    assert err["front"] < front_tol, err
    assert err["pe_vs_change"] < 1e-4, err
    assert err["ke"] < 1e-4, err
    return err

