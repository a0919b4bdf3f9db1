"""The allocation-free pair-pass entry point, checked against the regular one.

``tsph_wcsph_rhs_noalloc`` is for callers that own their input and output
buffers but cannot allocate device memory when they run the pair pass (their
host framework owns the memory pool, or their loop reserves memory once up
front).  It runs the same kernels as ``tsph_wcsph_rhs`` on the same inputs,
only on a fixed 16 MiB scratch array built into the library instead of a
caller's workspace; the kernels are deterministic (no floating-point atomics,
fixed summation orders), so every output must be bitwise equal to the regular
entry point's.

The array is shared by every call and keeps what the last call wrote.  The
test first fills it with a larger call, then runs, two calls in a row each
time, cases whose kernels use every region of the scratch: the split wall
loads, the compression regularisation (its per-particle sums and the carried
scalar it writes) and the free-surface closure (its known-pressure masks and
the Jacobi ping-pong buffer, with an even number of passes so that the result
comes back through that buffer).  Stale contents of the array would show up
as a difference.

This file is collected last on purpose: it runs after every other test.
"""
import ctypes
import math

import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(golden, tag, device, flags=None, diffusion=True):
    from tensorsph_b200.droplet_impact import Config, lattice_mass_unit, symmetric_rows
    g = golden("config1")
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * 2.0)
    cfg = Config(dx=0.02, sound_speed=c0, viscosity=1e-6, max_courant=0.25,
                 dt=0.25 * 1.3 * 0.02 / c0, wall_layers=3, density_diffusion=0.1,
                 wall_friction=0.5)
    pos = torch.from_numpy(g[f"{tag}_pos2"]).to(device).contiguous()
    vel = torch.from_numpy(g[f"{tag}_vel2"]).to(device).contiguous()
    mass = torch.from_numpy(g[f"{tag}_mass"]).to(device).contiguous()
    wall = torch.from_numpy(g[f"{tag}_wall"]).to(device).contiguous()
    pairs = torch.from_numpy(g[f"{tag}_pairs"]).to(device)
    n, nw = pos.shape[0], wall.shape[0]
    rowptr, entries = symmetric_rows(pairs, n + nw)
    from tensorsph_b200 import _lib
    h = cfg.h_factor * cfg.dx
    prm = _lib.WcsphParams()
    prm.dim, prm.dtype, prm.n_fluid, prm.n_wall = 2, _lib.dtype_code(pos.dtype), n, nw
    prm.flags = _lib.RHS_SPLIT if flags is None else flags
    prm.h, prm.sigma = h, 10.0 / (7.0 * math.pi * h * h)
    prm.rho0, prm.sound_speed, prm.gamma = cfg.rho0, cfg.sound_speed, cfg.gamma
    prm.gravity, prm.viscosity, prm.wall_friction = cfg.gravity, cfg.viscosity, cfg.wall_friction
    prm.diffusion_scale = 2.0 * cfg.density_diffusion * cfg.sound_speed * h if diffusion else 0.0
    prm.eigen_floor, prm.dt = 0.1, cfg.dt
    prm.wall_mass = lattice_mass_unit(cfg)
    # the compression regularisation ("reference_mean" normalisation, rule "all")
    prm.compression_rule, prm.compression_kref = 0, 1.0 / 1.0004
    # the free-surface closure: "interior" donors, two Jacobi passes
    prm.surface_donors, prm.surface_layers, prm.surface_threshold = 0, 2, 0.98
    inputs = dict(pos=pos, vel=vel, mass=mass, wall=wall, rowptr=rowptr, entries=entries)
    return prm, inputs


def _run(prm, t, noalloc):
    from tensorsph_b200 import _lib
    dev = t["pos"].device
    n, nw = prm.n_fluid, prm.n_wall
    fill = float("nan")   # every output the call owns must be written
    out = dict(rho=torch.full((n,), fill, dtype=t["pos"].dtype, device=dev),
               p=torch.full((n,), fill, dtype=t["pos"].dtype, device=dev),
               acc=torch.full((n, 2), fill, dtype=t["pos"].dtype, device=dev),
               reaction=torch.zeros((nw, 2), dtype=t["pos"].dtype, device=dev),
               face=torch.zeros(nw, dtype=t["pos"].dtype, device=dev),
               compression=torch.full((2,), fill, dtype=torch.float64, device=dev))
    split = prm.flags & _lib.RHS_SPLIT
    comp = prm.flags & _lib.RHS_COMPRESSION
    io = _lib.WcsphIO(t["pos"].data_ptr(), t["vel"].data_ptr(), t["mass"].data_ptr(),
                      t["wall"].data_ptr(), None, None, None, None, t["rowptr"].data_ptr(),
                      t["entries"].data_ptr(), out["rho"].data_ptr(), out["p"].data_ptr(),
                      out["acc"].data_ptr(), out["reaction"].data_ptr() if split else None,
                      out["face"].data_ptr() if split else None,
                      out["compression"].data_ptr() if comp else None)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    if noalloc:
        rc = L.tsph_wcsph_rhs_noalloc(ctypes.byref(prm), ctypes.byref(io), stream)
    else:
        ws = torch.empty(L.tsph_wcsph_workspace_bytes(ctypes.byref(prm)), dtype=torch.uint8,
                         device=dev)
        rc = L.tsph_wcsph_rhs(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                              stream)
    assert rc == 0, L.tsph_status_string(rc)
    torch.cuda.synchronize(dev)
    if not comp:
        del out["compression"]
    return out


def _dirty_scratch(gpu, golden):
    """A larger call than the checked ones, so that the shared array holds
    nonzero contents from another case before they run."""
    from tensorsph_b200 import _lib
    prm, t = _case(golden, "f64", gpu, flags=_lib.RHS_SPLIT | _lib.RHS_SURFACE_CLOSURE)
    prm.surface_layers = 3
    _run(prm, t, noalloc=True)


def test_noalloc_rhs_matches_regular_entry_point(gpu, golden):
    from tensorsph_b200 import _lib
    _dirty_scratch(gpu, golden)
    cases = (("f64", _lib.RHS_SPLIT, True), ("f32", _lib.RHS_SPLIT, True),
             ("f32", _lib.RHS_COMPRESSION, False), ("f64", _lib.RHS_COMPRESSION | _lib.RHS_SPLIT, False),
             ("f64", _lib.RHS_SURFACE_CLOSURE, True), ("f32", _lib.RHS_SURFACE_CLOSURE | _lib.RHS_SPLIT, True))
    for tag, flags, diffusion in cases:
        prm, t = _case(golden, tag, gpu, flags=flags, diffusion=diffusion)
        want = _run(prm, t, noalloc=False)
        for call in range(2):     # two calls in a row through the shared array
            got = _run(prm, t, noalloc=True)
            for key in want:
                assert torch.equal(got[key], want[key]), (tag, flags, call, key)
        assert not torch.isnan(want["rho"]).any() and not torch.isnan(want["acc"]).any()
        if flags & _lib.RHS_COMPRESSION:
            assert float(want["compression"][1]) > 0.0   # particles were compressed


def test_noalloc_rejects_oversized_calls(gpu):
    from tensorsph_b200 import _lib
    prm = _lib.WcsphParams()
    prm.dim, prm.dtype, prm.n_fluid, prm.n_wall = 3, _lib.F64, 2_000_000, 0
    io = _lib.WcsphIO()
    rc = _lib.lib().tsph_wcsph_rhs_noalloc(ctypes.byref(prm), ctypes.byref(io),
                                          torch.cuda.current_stream(gpu).cuda_stream)
    assert rc == _lib.ERR_CAPACITY


def test_empty_call_writes_identity_compression(gpu):
    """A call without fluid particles still writes the regulariser's result:
    1 / mean{S > 1} = 1 with a count of 0."""
    from tensorsph_b200 import _lib
    prm = _lib.WcsphParams()
    prm.dim, prm.dtype, prm.n_fluid, prm.n_wall = 2, _lib.F64, 0, 0
    prm.flags = _lib.RHS_COMPRESSION
    prm.compression_kref = 1.0
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=gpu)
    io = _lib.WcsphIO()
    io.compression_out = out.data_ptr()
    L = _lib.lib()
    stream = torch.cuda.current_stream(gpu).cuda_stream
    for fn in ("regular", "noalloc"):
        out.fill_(float("nan"))
        if fn == "regular":
            ws = torch.empty(max(L.tsph_wcsph_workspace_bytes(ctypes.byref(prm)), 256), dtype=torch.uint8,
                             device=gpu)
            rc = L.tsph_wcsph_rhs(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(), stream)
        else:
            rc = L.tsph_wcsph_rhs_noalloc(ctypes.byref(prm), ctypes.byref(io), stream)
        assert rc == 0
        torch.cuda.synchronize(gpu)
        assert out.tolist() == [1.0, 0.0], fn
