"""The allocation-free pair-pass entry point, checked against the regular one.

``tsph_wcsph_rhs_noalloc`` is for callers that own their input and output
buffers but cannot allocate device memory when they run the pair pass (their
host framework owns the memory pool, or their loop reserves memory once up
front).  It runs the same kernels as ``tsph_wcsph_rhs`` on a fixed 16 MiB
scratch array built into the library, so its results must match the regular
entry point's within the tolerances used for the rhs elsewhere (FP64 1e-12,
FP32 1e-5 on density and pressure / B, 1e-4 on acceleration).  Two calls in a
row, with different sizes and dtypes, also show that the contents one call
leaves in the shared array do not leak into the next.

This file is collected last on purpose: it runs after every other test.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(golden, tag, device):
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
    prm.flags = _lib.RHS_SPLIT
    prm.h, prm.sigma = h, 10.0 / (7.0 * math.pi * h * h)
    prm.rho0, prm.sound_speed, prm.gamma = cfg.rho0, cfg.sound_speed, cfg.gamma
    prm.gravity, prm.viscosity, prm.wall_friction = cfg.gravity, cfg.viscosity, cfg.wall_friction
    prm.diffusion_scale = 2.0 * cfg.density_diffusion * cfg.sound_speed * h
    prm.eigen_floor, prm.dt = 0.1, cfg.dt
    prm.wall_mass = lattice_mass_unit(cfg)
    inputs = dict(pos=pos, vel=vel, mass=mass, wall=wall, rowptr=rowptr, entries=entries)
    return prm, inputs


def _run(prm, t, noalloc):
    from tensorsph_b200 import _lib
    dev = t["pos"].device
    n, nw = prm.n_fluid, prm.n_wall
    out = dict(rho=torch.empty(n, dtype=t["pos"].dtype, device=dev),
               p=torch.empty(n, dtype=t["pos"].dtype, device=dev),
               acc=torch.empty((n, 2), dtype=t["pos"].dtype, device=dev),
               reaction=torch.empty((nw, 2), dtype=t["pos"].dtype, device=dev),
               face=torch.empty(nw, dtype=t["pos"].dtype, device=dev))
    io = _lib.WcsphIO(t["pos"].data_ptr(), t["vel"].data_ptr(), t["mass"].data_ptr(),
                      t["wall"].data_ptr(), None, None, None, None, t["rowptr"].data_ptr(),
                      t["entries"].data_ptr(), out["rho"].data_ptr(), out["p"].data_ptr(),
                      out["acc"].data_ptr(), out["reaction"].data_ptr(), out["face"].data_ptr())
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
    return {k: v.cpu().numpy() for k, v in out.items()}


def _close(a, b, scale, tol):
    return float(np.abs(a - b).max()) <= tol * scale


def test_noalloc_rhs_matches_regular_entry_point(gpu, golden):
    bulk = 1000.0 * (10.0 * math.sqrt(2.0 * 9.81 * 2.0)) ** 2 / 7.0
    # two calls in a row through the shared scratch: FP64 first, then FP32
    for tag, tol, tol_acc in (("f64", 1e-12, 1e-11), ("f32", 1e-5, 1e-4)):
        prm, t = _case(golden, tag, gpu)
        want = _run(prm, t, noalloc=False)
        got = _run(prm, t, noalloc=True)
        assert _close(got["rho"], want["rho"], np.abs(want["rho"]).max(), tol), tag
        assert _close(got["p"], want["p"], bulk, tol), tag
        assert _close(got["acc"], want["acc"], np.abs(want["acc"]).max(), tol_acc), tag
        assert _close(got["reaction"], want["reaction"],
                      max(np.abs(want["reaction"]).max(), 1e-30), tol_acc), tag
        assert _close(got["face"], want["face"], bulk, tol), tag


def test_noalloc_rejects_oversized_calls(gpu):
    from tensorsph_b200 import _lib
    prm = _lib.WcsphParams()
    prm.dim, prm.dtype, prm.n_fluid, prm.n_wall = 3, _lib.F64, 2_000_000, 0
    io = _lib.WcsphIO()
    rc = _lib.lib().tsph_wcsph_rhs_noalloc(ctypes.byref(prm), ctypes.byref(io),
                                          torch.cuda.current_stream(gpu).cuda_stream)
    assert rc == _lib.ERR_CAPACITY
