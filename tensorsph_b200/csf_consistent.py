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

With ``wall`` and ``contact_angle`` (csf_consistent.py:411-560,
contact_angle_isph.py:75-213): ``"rotate"`` turns the near-wall interface
normals toward the contact angle inside the fields (both colour gradients);
``"young"`` and ``"brackbill"`` leave the fields alone and add the wall-
adhesion traction ``C sigma delta_s w d`` to the force.  ``nearest_wall`` and
``apply_contact_angle_boundary`` are the standalone forms.  The nearest wall
particle is found from exact squared distances, the first of equals; the
reference's ``torch.cdist`` forms distances from dot products, which only
decides between wall particles at exactly equal distance.

All of it runs in the kernels of ``csrc/csf2.cu`` over symmetric pair rows,
in the dtype of the positions.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from .droplet_impact import symmetric_rows

__all__ = ["CSFState", "csf_fields", "surface_tension_acceleration", "nearest_wall",
           "apply_contact_angle_boundary", "CONTACT_ANGLE_REACH", "DEFAULT_TRACTION_CALIBRATION"]

CONTACT_ANGLE_REACH = 2.0
#: traction calibration C of the "young" / "brackbill" models
#: (contact_angle_isph.DEFAULT_TRACTION_CALIBRATION)
DEFAULT_TRACTION_CALIBRATION = 0.9611
_CONTACT = {"rotate": 1, "young": 2, "brackbill": 3}
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


def _options(curvature_scheme, delta_normalization):
    if delta_normalization not in _DELTA:
        raise ValueError(f"unknown delta_normalization {delta_normalization!r}; "
                         "expected ('legacy', 'local_range')")
    if curvature_scheme not in _CURVATURE:
        raise ValueError(f"unknown curvature_scheme {curvature_scheme!r}")


def _params(n, dtype, h, rho0=1.0, normal_smoothing=0, curvature_color_smoothing=0, curvature_scheme="mls",
            delta_normalization="legacy", curvature_stencil=4.0, sigma=0.0, n_wall=0, contact_model=0,
            contact_angle=0.0, contact_reach=CONTACT_ANGLE_REACH):
    prm = _lib.Csf2Params()
    prm.n, prm.dtype = int(n), _lib.dtype_code(dtype)
    prm.normal_smoothing, prm.color_smoothing = int(normal_smoothing), int(curvature_color_smoothing)
    prm.curvature, prm.delta_normalization = _CURVATURE[curvature_scheme], _DELTA[delta_normalization]
    prm.h, prm.rho0, prm.stencil, prm.sigma = float(h), float(rho0), float(curvature_stencil), float(sigma)
    prm.n_wall, prm.contact_model = int(n_wall), int(contact_model)
    prm.contact_angle, prm.contact_reach = float(contact_angle), float(contact_reach)
    prm.traction_calibration = DEFAULT_TRACTION_CALIBRATION
    return prm


def _wall(wall, dev, dtype):
    if wall is None:
        return None
    w = _lib.to_dev(wall.detach(), dev, dtype)
    if w.dim() != 2 or w.shape[1] != 2:
        raise ValueError("wall must have shape (M, 2)")
    return w


def _fields(pos, mass, pairs, h, rho0, normal_smoothing, curvature_scheme, curvature_stencil,
            curvature_color_smoothing, delta_normalization, wall=None, contact_angle=None,
            contact_reach=CONTACT_ANGLE_REACH):
    if pos.dim() != 2 or pos.shape[1] != 2:
        raise ValueError("csf_fields implements 2-D clouds")
    n, dtype = pos.shape[0], pos.dtype
    dev = _lib.cuda_device(pos)
    P = _lib.to_dev(pos.detach(), dev)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    W = _wall(wall, dev, dtype) if contact_angle is not None else None
    rotate = W is not None and W.shape[0] > 0
    rowptr, entries = symmetric_rows(_lib.to_dev(pairs, dev), n)
    out = [torch.empty(n, dtype=dtype, device=dev), torch.empty((n, 2), dtype=dtype, device=dev),
           torch.empty((n, 2), dtype=dtype, device=dev), torch.empty(n, dtype=dtype, device=dev),
           torch.empty(n, dtype=dtype, device=dev)]
    valid = torch.empty(n, dtype=torch.uint8, device=dev)
    prm = _params(n, dtype, h, rho0, normal_smoothing, curvature_color_smoothing, curvature_scheme,
                  delta_normalization, curvature_stencil, n_wall=W.shape[0] if rotate else 0,
                  contact_model=1 if rotate else 0, contact_angle=contact_angle or 0.0,
                  contact_reach=contact_reach)
    io = _lib.Csf2IO(P.data_ptr(), M.data_ptr(), rowptr.data_ptr(), entries.data_ptr(),
                     *[t.data_ptr() for t in out], valid.data_ptr(), W.data_ptr() if rotate else None)
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_csf2_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_csf2_fields(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                                  _lib.stream(dev)), "tsph_csf2_fields")
    return prm, out, ws, (P, M, W, valid, rowptr, entries)


def csf_fields(pos: torch.Tensor, mass: torch.Tensor, pairs: torch.Tensor, h: float, rho0: float,
               wall: torch.Tensor | None = None, contact_angle: float | None = None,
               contact_angle_reach: float = CONTACT_ANGLE_REACH, normal_smoothing: int = 2,
               curvature_scheme: str = "mls", curvature_stencil: float = 4.0,
               curvature_color_smoothing: int = 0, delta_normalization: str = "legacy",
               contact_angle_model: str = "rotate") -> CSFState:
    """Colour, its gradient, the outward normal, curvature and delta_s (with
    ``wall`` and ``contact_angle``: the near-wall normals turned toward it)."""
    _options(curvature_scheme, delta_normalization)
    out_device = pos.device
    _, (color, grad_c, normal, kappa, delta_s), _, _ = _fields(
        pos, mass, pairs, h, rho0, normal_smoothing, curvature_scheme, curvature_stencil,
        curvature_color_smoothing, delta_normalization, wall if contact_angle is not None else None,
        contact_angle, contact_angle_reach)
    return CSFState(color.to(out_device), grad_c.to(out_device), normal.to(out_device),
                    kappa.to(out_device), delta_s.to(out_device))


def surface_tension_acceleration(pos: torch.Tensor, density: torch.Tensor, mass: torch.Tensor,
                                 pairs: torch.Tensor, h: float, sigma: float, rho0: float | None = None,
                                 wall: torch.Tensor | None = None, contact_angle: float | None = None,
                                 contact_angle_reach: float = CONTACT_ANGLE_REACH,
                                 curvature_scheme: str = "mls", curvature_stencil: float = 4.0,
                                 delta_normalization: str = "legacy",
                                 contact_angle_model: str = "rotate") -> tuple[torch.Tensor, CSFState | None]:
    """CSF acceleration ``a = -sigma kappa delta_s n / rho`` and its fields;
    with ``wall`` and ``contact_angle`` the "rotate" boundary in the fields or
    the "young" / "brackbill" wall-adhesion traction in the force."""
    if sigma <= 0.0:
        return torch.zeros_like(pos), None
    model = contact_angle_model if contact_angle is not None else None
    if model is not None and model not in _CONTACT:
        raise ValueError(f"unknown contact_angle_model {contact_angle_model!r}")
    _options(curvature_scheme, delta_normalization)
    rho0 = float(rho0 if rho0 is not None else density.mean())
    out_device = pos.device
    if curvature_scheme != "mls" and pairs.numel() > 0:
        # the fit needs an arc: the list at the stencil, as the reference builds it
        from .neighbor_search import cell_linked_pairs
        pairs = cell_linked_pairs(pos, curvature_stencil * h)
    rotate = model in (None, "rotate")
    traction = model in ("young", "brackbill") and wall is not None
    prm, (color, grad_c, normal, kappa, delta_s), ws, (P, _, _, valid, _, _) = _fields(
        pos, mass, pairs, h, rho0, 2, curvature_scheme, curvature_stencil, 0, delta_normalization,
        wall if rotate else None, contact_angle if rotate else None, contact_angle_reach)
    dev, dtype = color.device, color.dtype
    R = _lib.to_dev(density.detach(), dev, dtype)
    ds_out = torch.empty_like(delta_s)
    acc = torch.empty_like(grad_c)
    prm.sigma = float(sigma)
    W = None
    if traction:
        W = _wall(wall, dev, dtype)
        if W.shape[0] == 0:
            raise ValueError("the wall-adhesion traction needs wall particles")
        prm.n_wall, prm.contact_model = W.shape[0], _CONTACT[model]
        prm.contact_angle = float(contact_angle)
        ws = _lib.workspace(_lib.lib().tsph_csf2_workspace_bytes(ctypes.byref(prm)), dev)
    io = _lib.Csf2IO(P.data_ptr(), None, None, None, color.data_ptr(), grad_c.data_ptr(), normal.data_ptr(),
                     kappa.data_ptr(), delta_s.data_ptr(), valid.data_ptr(), W.data_ptr() if traction else None)
    L = _lib.lib()
    _lib.check(L.tsph_csf2_acceleration(ctypes.byref(prm), ctypes.byref(io), R.data_ptr(), ds_out.data_ptr(),
                                        acc.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(dev)),
               "tsph_csf2_acceleration")
    state = CSFState(color.to(out_device), grad_c.to(out_device), normal.to(out_device),
                     kappa.to(out_device), ds_out.to(out_device))
    return acc.to(out_device), state


def nearest_wall(pos: torch.Tensor, wall_pos: torch.Tensor, chunk: int = 1024):
    """Distance to the nearest wall particle and the unit wall normal (from it
    to the particle); a particle on a wall particle takes the normalised mean
    direction of the others (csf_consistent.py:449-480).  ``chunk`` is the
    reference's memory knob and has no effect here."""
    n, dtype = pos.shape[0], pos.dtype
    if wall_pos.numel() == 0:
        raise ValueError("nearest_wall needs at least one wall particle")
    out_device = pos.device
    dev = _lib.cuda_device(pos)
    P = _lib.to_dev(pos.detach(), dev)
    W = _wall(wall_pos, dev, dtype)
    dist = torch.empty(n, dtype=dtype, device=dev)
    normal = torch.empty((n, 2), dtype=dtype, device=dev)
    if n == 0:
        return dist.to(out_device), normal.to(out_device)
    prm = _params(n, dtype, 1.0, n_wall=W.shape[0])
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_csf2_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_csf2_nearest_wall(ctypes.byref(prm), P.data_ptr(), W.data_ptr(), dist.data_ptr(),
                                        normal.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(dev)),
               "tsph_csf2_nearest_wall")
    return dist.to(out_device), normal.to(out_device)


def apply_contact_angle_boundary(grad_c: torch.Tensor, pos: torch.Tensor, wall_pos: torch.Tensor | None, h: float,
                                 theta: float, reach: float = CONTACT_ANGLE_REACH) -> torch.Tensor:
    """Young's contact angle on the colour gradient near a wall
    (csf_consistent.py:483-560): within ``reach * h`` of the wall the normal
    ``-grad c / |grad c|`` is blended (fully at the wall) toward
    ``cos(theta) n_wall + sin(theta) t``; ``|grad c|`` is kept."""
    if wall_pos is None or wall_pos.numel() == 0 or grad_c.numel() == 0:
        return grad_c.clone()
    if pos.dim() != 2 or pos.shape[1] != 2:
        raise ValueError("apply_contact_angle_boundary implements 2-D clouds")
    n, dtype = pos.shape[0], pos.dtype
    out_device = grad_c.device
    dev = _lib.cuda_device(pos)
    P = _lib.to_dev(pos.detach(), dev)
    W = _wall(wall_pos, dev, dtype)
    G = _lib.to_dev(grad_c.detach(), dev, dtype)
    out = torch.empty_like(G)
    prm = _params(n, dtype, h, n_wall=W.shape[0], contact_model=1, contact_angle=theta, contact_reach=reach)
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_csf2_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_csf2_contact_boundary(ctypes.byref(prm), P.data_ptr(), W.data_ptr(), G.data_ptr(),
                                            out.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(dev)),
               "tsph_csf2_contact_boundary")
    return out.to(out_device)
