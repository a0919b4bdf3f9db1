"""3-D CSF surface tension on the GPU (``tensorsph.threed.csf3``).

``csf_fields3`` and ``surface_tension_acceleration3`` keep the reference
signatures (threed/csf3.py:115-165, 220-238) and its ``CSFState3`` fields:

* colour ``c_i = sum_j V_j W_ij`` with ``V = m / rho0`` (or ``volume``);
* MLS matrix ``M_i = sum_j V_j (x_j - x_i) (x) grad_i W_ij``, replaced by the
  identity where ``|det M_i| <= 1e-6 median |det M|`` (``valid`` false);
* ``grad c = M^-1 sum_j V_j (c_j - c_i) grad_i W``, ``delta_s = |grad c|``,
  ``n = -grad c / |grad c|``;
* ``kappa = trace(S M^-1)``, ``S = sum_j V_j (n_j - n_i) (x) grad_i W``,
  zero where not valid;
* ``a = -sigma kappa delta_s n / rho`` on particles with
  ``delta_s > cutoff * max delta_s``.

The pair list becomes symmetric gather rows, and the passes run as the
kernels of ``csrc/csf3.cu``, in the dtype of the positions.  Separations use
the minimum image when ``box`` is given.  ``curvature="axisym"``
(csf3.py:168-220) replaces the curvature by the quadratic interface fit of
the meridional projection (r, z) within 4 h plus the azimuthal n_r / r; its
pair list must reach 4 h.  The reference documents that estimator as biased
on a cylinder and keeps it as a comparison arm; it is reproduced as it is.
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib
from ..droplet_impact import symmetric_rows
from .neighbors3 import _box_list

__all__ = ["csf_fields3", "surface_tension_acceleration3", "CSFState3", "CURVATURE_SCHEMES"]

#: The curvature schemes of the reference.
CURVATURE_SCHEMES = ("mls", "axisym")


class CSFState3:
    """The fields a 3-D CSF force is assembled from (all exposed for scoring)."""

    __slots__ = ("color", "grad_c", "normal", "kappa", "delta_s", "valid")

    def __init__(self, color, grad_c, normal, kappa, delta_s, valid):
        self.color = color
        self.grad_c = grad_c
        self.normal = normal
        self.kappa = kappa
        self.delta_s = delta_s
        self.valid = valid

    def surface_mask(self, fraction: float = 0.05) -> torch.Tensor:
        """Particles carrying a non-negligible share of the interface."""
        return self.delta_s > fraction * float(self.delta_s.max())

    def as_dict(self) -> dict:
        return {"color": self.color, "grad_c": self.grad_c, "normal": self.normal,
                "kappa": self.kappa, "delta_s": self.delta_s, "valid": self.valid}


def _params(n, dtype, h, rho0, box, sigma=0.0, cutoff=1.0e-3, curvature="mls"):
    prm = _lib.Csf3Params()
    prm.curvature = CURVATURE_SCHEMES.index(curvature)
    prm.n, prm.dtype = int(n), _lib.dtype_code(dtype)
    if box is not None:
        prm.periodic = 1
        for k, b in enumerate(_box_list(box, 3)):
            prm.box[k] = b
    prm.h, prm.rho0 = float(h), float(rho0)
    prm.sigma, prm.cutoff = float(sigma), float(cutoff)
    return prm


def csf_fields3(pos: torch.Tensor, mass: torch.Tensor, h: float, pairs: torch.Tensor, *,
                rho0: float, box=None, volume: torch.Tensor | None = None,
                curvature: str = "mls") -> CSFState3:
    """Colour, normal, curvature and delta function of a 3-D particle cloud."""
    if curvature not in CURVATURE_SCHEMES:
        raise ValueError(f"unknown curvature {curvature!r}; expected {CURVATURE_SCHEMES}")
    if pos.dim() != 2 or pos.shape[1] != 3:
        raise ValueError("csf_fields3 implements 3-D clouds")
    n = pos.shape[0]
    out_device, dtype = pos.device, pos.dtype
    dev = _lib.cuda_device(pos)
    P = _lib.to_dev(pos.detach(), dev)
    M = _lib.to_dev(mass.detach(), dev, dtype)
    Vol = None if volume is None else _lib.to_dev(volume.detach(), dev, dtype)
    rowptr, entries = symmetric_rows(_lib.to_dev(pairs, dev), n)
    color = torch.empty(n, dtype=dtype, device=dev)
    grad_c = torch.empty((n, 3), dtype=dtype, device=dev)
    normal = torch.empty((n, 3), dtype=dtype, device=dev)
    kappa = torch.empty(n, dtype=dtype, device=dev)
    delta_s = torch.empty(n, dtype=dtype, device=dev)
    valid = torch.empty(n, dtype=torch.uint8, device=dev)
    prm = _params(n, dtype, h, rho0, box, curvature=curvature)
    io = _lib.Csf3IO(P.data_ptr(), M.data_ptr(), 0 if Vol is None else Vol.data_ptr(),
                     rowptr.data_ptr(), entries.data_ptr(), color.data_ptr(), grad_c.data_ptr(),
                     normal.data_ptr(), kappa.data_ptr(), delta_s.data_ptr(), valid.data_ptr())
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_csf3_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_csf3_fields(ctypes.byref(prm), ctypes.byref(io), ws.data_ptr(), ws.numel(),
                                  _lib.stream(dev)), "tsph_csf3_fields")
    return CSFState3(color.to(out_device), grad_c.to(out_device), normal.to(out_device),
                     kappa.to(out_device), delta_s.to(out_device), valid.bool().to(out_device))


def surface_tension_acceleration3(csf: CSFState3, rho: torch.Tensor, sigma: float,
                                  cutoff: float = 1.0e-3) -> torch.Tensor:
    """``a_i = -sigma kappa_i delta_s_i n_i / rho_i`` (force per unit mass)."""
    if sigma == 0.0:
        return torch.zeros_like(csf.normal)
    out_device, dtype = csf.normal.device, csf.normal.dtype
    dev = _lib.cuda_device(csf.normal)
    n = csf.normal.shape[0]
    Nr = _lib.to_dev(csf.normal.detach(), dev)
    K = _lib.to_dev(csf.kappa.detach(), dev, dtype)
    D = _lib.to_dev(csf.delta_s.detach(), dev, dtype)
    R = _lib.to_dev(rho.detach(), dev, dtype)
    acc = torch.empty((n, 3), dtype=dtype, device=dev)
    prm = _params(n, dtype, 1.0, 1.0, None, sigma=sigma, cutoff=cutoff)
    L = _lib.lib()
    ws = _lib.workspace(L.tsph_csf3_workspace_bytes(ctypes.byref(prm)), dev)
    _lib.check(L.tsph_csf3_acceleration(ctypes.byref(prm), Nr.data_ptr(), K.data_ptr(), D.data_ptr(),
                                        R.data_ptr(), acc.data_ptr(), ws.data_ptr(), ws.numel(),
                                        _lib.stream(dev)), "tsph_csf3_acceleration")
    return acc.to(out_device)
