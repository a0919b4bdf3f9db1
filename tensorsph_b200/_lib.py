"""ctypes binding of ``libtsph_b200.so`` (the C ABI in ``include/tsph.h``).

Loading fails loudly: there is no CPU fallback anywhere in this package.  Every
call passes raw device pointers of torch tensors plus torch's current CUDA
stream, so the library is stream-ordered with the caller's work and all
memory (outputs and workspaces) comes from torch's caching allocator.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_int64, c_void_p
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libtsph_b200.so"

F32, F64 = 0, 1

OK = 0
ERR_ARG, ERR_NONFINITE, ERR_CUDA, ERR_WORKSPACE, ERR_CAPACITY = 1, 2, 3, 4, 5
ERR_UNSUPPORTED, ERR_INDEX, ERR_GRID, ERR_STATE, ERR_TIMEOUT = 6, 7, 8, 9, 10

RHS_RENORMALIZE, RHS_BOUNDARY_DENSITY, RHS_SPLIT, RHS_WALL_SELF, RHS_WRAP_X = 1, 2, 4, 8, 16
RHS_COMPRESSION, RHS_SURFACE_CLOSURE = 32, 64


class Grid(ctypes.Structure):
    _fields_ = [("n", c_int64), ("dim", c_int64), ("dtype", c_int64), ("periodic", c_int64),
                ("cutoff", c_double), ("box", c_double * 3), ("width", c_double * 3),
                ("ncell", c_int64 * 3), ("origin", c_int64 * 3), ("total_cells", c_int64),
                ("dense", c_int64), ("key_bits", c_int64), ("workspace_bytes", c_int64)]


class WcsphParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("dim", "dtype", "n_fluid", "n_wall", "flags",
                                       "diffusion_form")] + \
               [(k, c_double) for k in ("h", "sigma", "rho0", "sound_speed", "gamma", "gravity",
                                        "viscosity", "wall_friction", "diffusion_scale",
                                        "eigen_floor", "dt", "wall_mass", "wrap_width",
                                        "lattice_sum")] + \
               [("compression_rule", c_int64), ("compression_kref", c_double),
                ("surface_donors", c_int64), ("surface_layers", c_int64),
                ("surface_threshold", c_double)]


class WcsphIO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "vel", "mass", "wall", "wall_vel", "wall_accel",
                                        "nu_field", "density_offset", "rowptr", "entries", "rho",
                                        "pressure", "acc", "reaction", "face_pressure",
                                        "compression_out")]


class ThreedParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("dtype", "n", "n_fluid", "has_gravity", "periodic",
                                       "renormalise", "wall_model", "viscous_order",
                                       "diffusion_form")] + \
               [(k, c_double) for k in ("h", "rho0", "sound_speed", "gamma", "viscosity",
                                        "diffusion", "dt", "eigen_floor")] + \
               [("gravity", c_double * 3), ("box", c_double * 3)]


class ThreedIO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "vel", "mass", "rowptr", "entries", "acc", "rho",
                                        "pressure")]


class Csf3Params(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("n", "dtype", "periodic")] + \
               [("box", c_double * 3)] + \
               [(k, c_double) for k in ("h", "rho0", "sigma", "cutoff")] + \
               [("curvature", c_int64)]


class Csf3IO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "mass", "volume", "rowptr", "entries", "color",
                                        "grad_c", "normal", "kappa", "delta_s", "valid")]


class Csf2Params(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("n", "dtype", "normal_smoothing", "color_smoothing", "curvature",
                                       "delta_normalization", "n_wall", "contact_model")] + \
               [(k, c_double) for k in ("h", "rho0", "stencil", "sigma", "contact_angle", "contact_reach",
                                        "traction_calibration")]


class Csf2IO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "mass", "rowptr", "entries", "color", "grad_c", "normal",
                                        "kappa", "delta_s", "valid", "wall")]


class TvcParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("n_total", "n_fluid", "dim", "dtype", "has_ratio", "limiter",
                                       "has_scope_tol", "has_max_shift")] + \
               [(k, c_double) for k in ("h", "h_ref", "h_ratio_scale", "wall_factor", "alpha", "slope",
                                        "scope_tol", "max_shift")]


class TvcIO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "volume", "h_ratio", "correction", "rowptr", "entries",
                                        "gradient", "squared", "limiter_in", "active", "limiter_out",
                                        "shift", "clipped")]


class ShiftParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("dim", "dtype", "n")] + \
               [(k, c_double) for k in ("h", "sigma", "magnitude", "cap", "free_surface",
                                        "c_reference")]


class ShiftIO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "volume", "rowptr", "entries", "out_pos",
                                        "concentration", "grad", "normal", "shift",
                                        "free_surface", "c_reference")]


class ClampParams(ctypes.Structure):
    _fields_ = [("dim", c_int64), ("dtype", c_int64), ("n", c_int64),
                ("lo", c_double * 3), ("hi", c_double * 3), ("tolerance", c_double),
                ("has_obstacle", c_int64), ("ob_lo", c_double * 3), ("ob_hi", c_double * 3),
                ("ob_eps", c_double)]


class DeltaPlusParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("dtype", "n_fluid", "n_wall")] + \
               [(k, c_double) for k in ("dx", "sound_speed", "reference_speed", "dt", "rho0",
                                        "gravity", "viscosity", "diffusion", "alpha")] + \
               [("dim", c_int64)]


class DeltaPlusIO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "vel", "density", "mass", "wall", "wall_vel",
                                        "wall_normal", "rowptr", "entries", "out_pos", "out_vel",
                                        "out_density", "acc", "reaction", "shift", "status_out")]


class MeterParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("dim", "dtype", "n", "periodic")] + \
               [(k, c_double) for k in ("rho0", "sound_speed", "gamma")] + \
               [("origin", c_double * 3), ("box", c_double * 3)]


class MeterIO(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("pos", "vel", "mass", "rho", "out")]


class EngineParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("max_fluid", "max_wall", "max_obstacle", "max_cells",
                                       "max_cases", "max_neighbors", "diag_ring",
                                       "max_fit_neighbors")]


class CaseParams(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("dim", "n_fluid", "n_wall", "n_obstacle", "shift_every",
                                       "has_obstacle")] + \
               [(k, c_double) for k in ("h", "rho0", "sound_speed", "gamma", "gravity",
                                        "viscosity", "wall_friction", "diffusion_scale", "dt",
                                        "wall_mass", "skin")] + \
               [("box_hi", c_double * 3), ("tolerance", c_double), ("ob_lo", c_double * 3),
                ("ob_hi", c_double * 3), ("ob_eps", c_double), ("shift_strength", c_double),
                ("shift_limit", c_double), ("shift_free_surface", c_double),
                ("shift_vref_floor", c_double), ("grid_lo", c_double * 3),
                ("grid_hi", c_double * 3), ("surface_tension", c_double),
                ("periodic_box", c_double), ("tvc_every", c_int64), ("tvc_alpha", c_double),
                ("tvc_scope_tol", c_double), ("tvc_max_shift", c_double),
                ("first_step", c_int64), ("tvc_slope", c_double), ("tvc_wall_volume", c_double),
                ("tvc_bulk_c", c_double), ("csf_curvature", c_int64), ("csf_delta_normalization", c_int64),
                ("csf_contact_model", c_int64), ("csf_contact_angle", c_double), ("csf_contact_reach", c_double),
                ("csf_wall_area", c_double), ("csf_traction_calibration", c_double),
                ("adaptive_dt", c_int64), ("courant_h", c_double), ("dt_limit", c_double),
                ("dt_growth", c_double), ("dt_safety", c_double), ("target_time", c_double),
                ("shift_vref_given", c_int64), ("shift_vref", c_double),
                ("diffusion_form", c_int64), ("diffusion_eigen_floor", c_double),
                ("density_renormalization", c_int64), ("lattice_kernel_sum", c_double),
                ("boundary_consistent_density", c_int64),
                ("start_elapsed", c_double), ("start_dt", c_double),
                ("compression", c_int64), ("compression_rule", c_int64),
                ("compression_normalization", c_int64), ("surface_closure", c_int64),
                ("surface_threshold", c_double), ("surface_donors", c_int64), ("surface_layers", c_int64)]


_SIGNATURES = {
    "tsph_abi_version": (c_int, []),
    "tsph_status_string": (ctypes.c_char_p, [c_int]),
    "tsph_grid_plan_scratch_bytes": (c_int64, []),
    "tsph_grid_plan": (c_int, [c_void_p, c_int64, c_int64, c_int64, c_double, c_void_p, c_void_p,
                               POINTER(Grid), c_void_p]),
    "tsph_grid_build": (c_int, [c_void_p, POINTER(Grid), c_void_p, c_int64, c_void_p, c_void_p]),
    "tsph_pairs_count": (c_int, [c_void_p, POINTER(Grid), c_int64, c_void_p, c_int64,
                                 POINTER(c_int64), POINTER(c_int64), c_void_p]),
    "tsph_pairs_emit_workspace_bytes": (c_int64, [c_int64, c_int64]),
    "tsph_pairs_emit": (c_int, [c_void_p, POINTER(Grid), c_int64, c_void_p, c_int64, c_void_p,
                                c_int64, c_void_p, c_int64, c_void_p]),
    "tsph_brute_workspace_bytes": (c_int64, [c_int64]),
    "tsph_brute_pairs_count": (c_int, [c_void_p, c_int64, c_int64, c_int64, c_double, c_void_p,
                                       c_int64, POINTER(c_int64), c_void_p]),
    "tsph_brute_pairs_emit": (c_int, [c_void_p, c_int64, c_int64, c_int64, c_double, c_void_p,
                                      c_int64, c_void_p, c_int64, c_void_p]),
    "tsph_max_displacement": (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_int64, c_void_p,
                                      c_void_p, c_void_p]),
    "tsph_csr_workspace_bytes": (c_int64, [c_int64, c_int64]),
    "tsph_csr_from_pairs": (c_int, [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p,
                                    c_int64, c_void_p]),
    "tsph_wcsph_workspace_bytes": (c_int64, [POINTER(WcsphParams)]),
    "tsph_wcsph_rhs": (c_int, [POINTER(WcsphParams), POINTER(WcsphIO), c_void_p, c_int64,
                               c_void_p]),
    "tsph_wcsph_rhs_noalloc": (c_int, [POINTER(WcsphParams), POINTER(WcsphIO), c_void_p]),
    "tsph_threed_workspace_bytes": (c_int64, [POINTER(ThreedParams)]),
    "tsph_threed_accelerations": (c_int, [POINTER(ThreedParams), POINTER(ThreedIO), c_void_p,
                                          c_int64, c_void_p]),
    "tsph_csf2_workspace_bytes": (c_int64, [POINTER(Csf2Params)]),
    "tsph_csf2_fields": (c_int, [POINTER(Csf2Params), POINTER(Csf2IO), c_void_p, c_int64, c_void_p]),
    "tsph_csf2_acceleration": (c_int, [POINTER(Csf2Params), POINTER(Csf2IO), c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_int64, c_void_p]),
    "tsph_csf2_nearest_wall": (c_int, [POINTER(Csf2Params), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_int64, c_void_p]),
    "tsph_csf2_contact_boundary": (c_int, [POINTER(Csf2Params), c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_int64, c_void_p]),
    "tsph_tvc_gradient": (c_int, [POINTER(TvcParams), POINTER(TvcIO), c_void_p]),
    "tsph_tvc_shift": (c_int, [POINTER(TvcParams), POINTER(TvcIO), c_void_p]),
    "tsph_csf3_workspace_bytes": (c_int64, [POINTER(Csf3Params)]),
    "tsph_csf3_fields": (c_int, [POINTER(Csf3Params), POINTER(Csf3IO), c_void_p, c_int64, c_void_p]),
    "tsph_csf3_acceleration": (c_int, [POINTER(Csf3Params), c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_int64, c_void_p]),
    "tsph_shift_workspace_bytes": (c_int64, [POINTER(ShiftParams)]),
    "tsph_shift_positions": (c_int, [POINTER(ShiftParams), POINTER(ShiftIO), c_void_p, c_int64,
                                     c_void_p]),
    "tsph_quantile_workspace_bytes": (c_int64, [c_int64]),
    "tsph_quantile": (c_int, [c_void_p, c_int64, c_int64, c_double, c_void_p, c_void_p, c_int64,
                              c_void_p]),
    "tsph_euler_clamp": (c_int, [POINTER(ClampParams), c_void_p, c_void_p, c_void_p, c_double,
                                 c_void_p, c_void_p]),
    "tsph_delta_plus_workspace_bytes": (c_int64, [POINTER(DeltaPlusParams)]),
    "tsph_delta_plus_step": (c_int, [POINTER(DeltaPlusParams), POINTER(DeltaPlusIO), c_void_p,
                                     c_int64, c_void_p]),
    "tsph_meters_workspace_bytes": (c_int64, []),
    "tsph_meters": (c_int, [POINTER(MeterParams), POINTER(MeterIO), c_void_p, c_int64, c_void_p]),
    "tsph_mode_amplitude": (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_double, c_int64,
                                    c_void_p, c_int64, c_void_p, c_void_p]),
    "tsph_kick_drift": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_double,
                                c_int64, c_void_p, c_void_p]),
    "tsph_internal_energy": (c_int, [c_void_p, c_int64, c_int64, c_double, c_double, c_double,
                                     c_void_p, c_void_p]),
    "tsph_engine_bytes": (c_int64, [POINTER(EngineParams)]),
    "tsph_engine_case_cells": (c_int64, [POINTER(CaseParams)]),
    "tsph_engine_create": (c_int, [POINTER(EngineParams), c_void_p, c_int64, c_void_p, c_void_p]),
    "tsph_engine_add_case": (c_int, [c_void_p, POINTER(CaseParams), c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, POINTER(c_int64)]),
    "tsph_engine_remove_case": (c_int, [c_void_p, c_int64, c_void_p]),
    "tsph_engine_step": (c_int, [c_void_p, c_int64, c_void_p]),
    "tsph_engine_step_eager": (c_int, [c_void_p, c_int64, c_void_p]),
    "tsph_engine_step_timed": (c_int, [c_void_p, c_void_p, POINTER(ctypes.c_float),
                                       POINTER(c_int64)]),
    "tsph_engine_graph_kernels": (c_int, [c_void_p, POINTER(c_int64)]),
    "tsph_engine_read": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p]),
    "tsph_engine_diag": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_int64, c_void_p]),
    "tsph_engine_status": (c_int, [c_void_p, c_int64, c_void_p, c_void_p]),
    "tsph_engine_clock": (c_int, [c_void_p, c_int64, c_void_p, c_void_p]),
    "tsph_engine_usage": (c_int, [c_void_p, c_void_p]),
    "tsph_engine_row_entries": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tsph_engine_graph_stats": (c_int, [c_void_p, c_void_p]),
    "tsph_engine_set_block": (c_int, [c_void_p, c_int64]),
    "tsph_engine_set_batch": (c_int, [c_void_p, c_int64]),
    "tsph_engine_destroy": (c_int, [c_void_p]),
    "tsph_probe_fma": (c_int, [c_void_p, c_int64, c_int64, c_int64, c_int64, c_void_p]),
    "tsph_probe_fma_flops": (c_int64, [c_int64, c_int64, c_int64, c_int64]),
    "tsph_probe_copy": (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_void_p]),
}

EXPORTED = tuple(_SIGNATURES)

_LIB = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m tensorsph_b200.build` "
                "(the B200 particle pass has no CPU fallback)")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


class TsphError(RuntimeError):
    pass


def check(code: int, what: str) -> None:
    if code == OK:
        return
    msg = f"{what}: {lib().tsph_status_string(code).decode()} (code {code})"
    if code in (ERR_ARG, ERR_NONFINITE, ERR_INDEX, ERR_GRID):
        raise ValueError(msg)
    if code == ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if code == ERR_STATE:
        raise FloatingPointError(msg)
    raise TsphError(msg)


def cuda_device(like: torch.Tensor | None = None) -> torch.device:
    """The CUDA device a call runs on (the input's when it is already there)."""
    if like is not None and like.is_cuda:
        return like.device
    if not torch.cuda.is_available():
        raise RuntimeError("tensorsph_b200 needs a CUDA device (B200); no CPU fallback exists")
    return torch.device("cuda", torch.cuda.current_device())


def stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return F32
    if dtype == torch.float64:
        return F64
    raise TypeError(f"positions must be float32 or float64, got {dtype}")


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def to_dev(t: torch.Tensor | None, device: torch.device, dtype: torch.dtype | None = None):
    if t is None:
        return None
    return t.to(device=device, dtype=dtype or t.dtype).contiguous()
