"""Transport-velocity correction on the GPU against the reference's own
output (tests/golden/tvc.npz) and the oracle.

Tolerances, relative to each field's largest magnitude: FP64 1e-12, FP32 2e-5
(the device sums each particle's row in a fixed order where the reference
scatters with index_add).  The clipped fraction is exact.
"""
import numpy as np
import pytest
import torch

from tests.test_oracle_golden import _tvc_kwargs

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_tvc_matches_reference(golden, gpu):
    from tensorsph_b200 import transport_velocity_correction as tv
    g = golden("tvc")
    for k in range(int(g["count"])):
        kw = _tvc_kwargs(g, k)
        if "active" in kw:
            kw["active"] = _t(kw["active"])
        if "h_ratio" in kw:
            kw["h_ratio"] = _t(kw["h_ratio"])
        if int(g[f"c{k}_limiter_tl"]):
            kw["limiter"] = tv.truncated_linear(100.0)
        pos = g[f"c{k}_pos"]
        res = tv.transport_velocity_correction(_t(pos), _t(g[f"c{k}_volume"]), float(g[f"c{k}_h"]),
                                               pairs=_t(g[f"c{k}_pairs"]), **kw)
        tol = 1e-12 if pos.dtype == np.float64 else 2e-5
        for name in ("gradient_integral", "shift", "squared_norm", "limiter"):
            ref = g[f"c{k}_{name}"]
            got = getattr(res, name).cpu().numpy()
            assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (k, name)
        assert res.clipped == float(g[f"c{k}_clipped"]), k


def test_tvc_custom_limiter_and_correction_match_oracle(golden, gpu):
    """A user limiter (evaluated on the device tensor of h_ref^2 |g|^2) and
    kernel_gradient_integral with kernel-correction factors and another wall
    factor, against the oracle."""
    from oracle import tvc as otv
    from tensorsph_b200 import transport_velocity_correction as tv
    g = golden("tvc")
    for k in (0, 5):
        pos, vol, pairs = g[f"c{k}_pos"], g[f"c{k}_volume"], g[f"c{k}_pairs"]
        h, nw = float(g[f"c{k}_h"]), int(g[f"c{k}_n_wall"])
        lim = lambda m: torch.sqrt(torch.clamp(m, max=1.0))
        res = tv.transport_velocity_correction(_t(pos), _t(vol), h, pairs=_t(pairs), wall_count=nw,
                                               limiter=lim, max_shift=1e-4)
        ref = otv.transport_velocity_correction(pos, vol, h, pairs, wall_count=nw, max_shift=1e-4)
        # the oracle without a limiter, rescaled by the same factor
        fac = np.sqrt(np.minimum((h * h) * ref["squared_norm"], 1.0))
        assert np.abs(res.limiter.cpu().numpy() - fac).max() <= 1e-12
        c = 0.9 + 0.2 * np.random.default_rng(k).random(pos.shape[0])
        got = tv.kernel_gradient_integral(_t(pos), _t(vol), h, pairs=_t(pairs), wall_count=nw, wall_factor=1.5,
                                          correction=_t(c)).cpu().numpy()
        want = otv.kernel_gradient_integral(pos, vol, h, pairs, wall_count=nw, wall_factor=1.5, correction=c)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_tvc_without_pairs_searches_them(golden, gpu):
    """pairs=None: the device cell search at 2h (2h / min h_ratio) gives the
    result of the explicit pair list."""
    from tensorsph_b200 import transport_velocity_correction as tv
    g = golden("tvc")
    for k in (0, 4):
        kw = _tvc_kwargs(g, k)
        if "h_ratio" in kw:
            kw["h_ratio"] = _t(kw["h_ratio"])
        a = tv.transport_velocity_correction(_t(g[f"c{k}_pos"]), _t(g[f"c{k}_volume"]), float(g[f"c{k}_h"]), **kw)
        ref = g[f"c{k}_shift"]
        assert np.abs(a.shift.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max(), k
