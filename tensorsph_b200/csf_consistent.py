"""2-D CSF surface tension on the GPU (``tensorsph.csf_consistent``).

``csf_fields`` and ``surface_tension_acceleration`` keep the reference
signatures and the ``CSFState`` fields (csf_consistent.py:75-446):

* colour ``c = clip(sum_j V_j W_ij + V_i W(0), 0, 1)``, ``V = m / rho0``;
* MLS gradient ``M^-T sum_j V_j (c_j - c_i) grad_i W`` with the identity
  for ``|det M| <= 1e-4 median |det M|``;
* normal ``-grad c / |grad c|`` with ``normal_smoothing`` Shepard passes;
* curvature ``div n`` (``"mls"``), the weighted quadratic interface fit over
  ``curvature_stencil * h`` (``"fit_quadratic"``, csf_curvature.py:78-166) or
  the Pratt circle fit with the same weights (``"fit_circle"``, :179-213),
  the MLS value where a fit is not regular; ``div n`` optionally from the
  normal of a Shepard-smoothed colour (``curvature_color_smoothing``);
* ``delta_s = 2 |grad c|`` (``"legacy"``) or ``|grad c| / clip(max c - min c,
  0.2, 1)`` over the neighbourhood (``"local_range"``);
* ``a = -sigma kappa delta_s n / rho`` with ``delta_s = 0`` where
  ``|grad c| <= 1e-3 max |grad c|``; with a fit the pair list is rebuilt at
  the stencil, as the reference does.

All of it runs in the kernels of ``csrc/csf2.cu`` over symmetric pair rows,
in the dtype of the positions.  Contact angles (``wall`` + ``contact_angle``)
are not built and raise ``NotImplementedError``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from .droplet_impact import symmetric_rows

__all__ = ["CSFState", "csf_fields", "surface_tension_acceleration", "CONTACT_ANGLE_REACH"]

CONTACT_ANGLE_REACH = 2.0
_CURVATURE = {"mls": 0, "fit_quadratic": 1, "fit_circle": 2}
_DELTA = {"legacy": 0, "local_range": 1}


@dataclass
class CSFState:
    """The fields the CSF force is assembled from (all exposed for scoring)."""

    color: torch.Tensor
    grad_c: torch.Tensor
    normal: torch.Tensor
    kappa: torch.Tensor
    delta_s: torch.Tensor

    def surface_mask(self, fraction: float = 0.05) -> torch.Tensor:
        """Particles carrying a non-negligible share of the interface."""
        cut = fraction * float(self.delta_s.max())
        return self.delta_s > cut


def _options(curvature_scheme, delta_normalization, wall, contact_angle):
    if delta_normalization not in _DELTA:
        raise ValueError(f"unknown delta_normalization {delta_normalization!r}; "
                         "expected ('legacy', 'local_range')")
    if curvature_scheme not in _CURVATURE:
        raise ValueError(f"unknown curvature_scheme {curvature_scheme!r}")
    if wall is not None and contact_angle is not None:
        raise NotImplementedError("the contact-angle boundary is not part of the device CSF")


def _params(n, dtype, h, rho0, normal_smoothing, curvature_color_smoothing, curvature_scheme,
            delta_normalization, curvature_stencil, sigma=0.0):
    prm = _lib.Csf2Params()
    prm.n, prm.dtype = int(n), _lib.dtype_code(dtype)
    prm.normal_smoothing, prm.color_smoothing = int(normal_smoothing), int(curvature_color_smoothing)
    prm.curvature, prm.delta_normalization = _CURVATURE[curvature_scheme], _DELTA[delta_normalization]
    prm.h, prm.rho0, prm.stencil, prm.sigma = float(h), float(rho0), float(curvature_stencil), float(sigma)
    return prm


def _fields(pos, mass, pairs, h, rho0, normal_smoothing, curvature_scheme, curvature_stencil,
            curvature_color_smoothing, delta_normalization):
    if pos.dim() != 2 or pos.shape[1] != 2:
        raise ValueError("csf_fields implements 2-D clouds")
    n, dtype = pos.shape[0], pos.dtype
    dev = _lib.cuda_device(pos)
    P = _lib.to_dev(pos.detach(), dev)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    rowptr, entries = symmetric_rows(_lib.to_dev(pairs, dev), n)
    out = [torch.empty(n, dtype=dtype, device=dev), torch.empty((n, 2), dtype=dtype, device=dev),
           torch.empty((n, 2), dtype=dtype, device=dev), torch.empty(n, dtype=dtype, device=dev),
           torch.empty(n, dtype=dtype, device=dev)]
    valid = torch.empty(n, dtype=torch.uint8, device=dev)
    prm = _params(n, dtype, h, rho0, normal_smoothing, curvature_color_smoothing, curvature_scheme,
                  delta_normalization, curvature_stencil)
    io = _lib.Csf2IO(P.data_ptr(), M.data_ptr(), rowptr.data_ptr(), entries.data_ptr(),
                     *[t.data_ptr() for t in out], valid.data_ptr())
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_csf2_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_csf2_fields(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                                  _lib.stream(dev)), "tsph_csf2_fields")
    return prm, out, ws


def csf_fields(pos: torch.Tensor, mass: torch.Tensor, pairs: torch.Tensor, h: float, rho0: float,
               wall: torch.Tensor | None = None, contact_angle: float | None = None,
               contact_angle_reach: float = CONTACT_ANGLE_REACH, normal_smoothing: int = 2,
               curvature_scheme: str = "mls", curvature_stencil: float = 4.0,
               curvature_color_smoothing: int = 0, delta_normalization: str = "legacy",
               contact_angle_model: str = "rotate") -> CSFState:
    """Colour, its gradient, the outward normal, curvature and delta_s."""
    _options(curvature_scheme, delta_normalization, wall, contact_angle)
    out_device = pos.device
    _, (color, grad_c, normal, kappa, delta_s), _ = _fields(
        pos, mass, pairs, h, rho0, normal_smoothing, curvature_scheme, curvature_stencil,
        curvature_color_smoothing, delta_normalization)
    return CSFState(color.to(out_device), grad_c.to(out_device), normal.to(out_device),
                    kappa.to(out_device), delta_s.to(out_device))


def surface_tension_acceleration(pos: torch.Tensor, density: torch.Tensor, mass: torch.Tensor,
                                 pairs: torch.Tensor, h: float, sigma: float, rho0: float | None = None,
                                 wall: torch.Tensor | None = None, contact_angle: float | None = None,
                                 contact_angle_reach: float = CONTACT_ANGLE_REACH,
                                 curvature_scheme: str = "mls", curvature_stencil: float = 4.0,
                                 delta_normalization: str = "legacy",
                                 contact_angle_model: str = "rotate") -> tuple[torch.Tensor, CSFState | None]:
    """CSF acceleration ``a = -sigma kappa delta_s n / rho`` and its fields."""
    if sigma <= 0.0:
        return torch.zeros_like(pos), None
    if contact_angle is not None and contact_angle_model not in ("rotate", "young", "brackbill"):
        raise ValueError(f"unknown contact_angle_model {contact_angle_model!r}")
    _options(curvature_scheme, delta_normalization, wall, contact_angle)
    rho0 = float(rho0 if rho0 is not None else density.mean())
    out_device = pos.device
    if curvature_scheme != "mls" and pairs.numel() > 0:
        # the fit needs an arc: the list at the stencil, as the reference builds it
        from .neighbor_search import cell_linked_pairs
        pairs = cell_linked_pairs(pos, curvature_stencil * h)
    prm, (color, grad_c, normal, kappa, delta_s), ws = _fields(
        pos, mass, pairs, h, rho0, 2, curvature_scheme, curvature_stencil, 0, delta_normalization)
    dev, dtype = color.device, color.dtype
    R = _lib.to_dev(density.detach(), dev, dtype)
    ds_out = torch.empty_like(delta_s)
    acc = torch.empty_like(grad_c)
    prm.sigma = float(sigma)
    L = _lib.lib()
    _lib.check(L.tsph_csf2_acceleration(ctypes.byref(prm), grad_c.data_ptr(), normal.data_ptr(),
                                        kappa.data_ptr(), delta_s.data_ptr(), R.data_ptr(), ds_out.data_ptr(),
                                        acc.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(dev)),
               "tsph_csf2_acceleration")
    state = CSFState(color.to(out_device), grad_c.to(out_device), normal.to(out_device),
                     kappa.to(out_device), ds_out.to(out_device))
    return acc.to(out_device), state
