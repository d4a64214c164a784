"""Drop-in for ``GlobalMatrix.gmm_torch`` (``gmm_torch.py:229-380``).

``gmm_reflectivity_torch`` has the reference's signature; its value comes from the
block-Riccati GMM kernel (``kr_gmm_reflectivity``).  The reference differentiates through
``torch.linalg.solve``; here the derivative is the hand-written Kennett adjoint of the same
function R(alpha, beta, rho, h) (the two methods compute one reflectivity, equal to ~1e-10),
attached so that autograd, ``torch.func.jacrev`` and ``torch.func.hessian`` see the GMM value
with the adjoint's derivative.  ``gmm_jacobian`` and ``gmm_hessian`` are the Kennett
``jacobian`` / ``hessian`` of this package for the same reason.
"""

from __future__ import annotations

import torch

from . import device as D
from .kennett_torch import _device_for, _needs_grad, hessian, jacobian, kennett_reflectivity_torch

__all__ = ["gmm_reflectivity_torch", "gmm_jacobian", "gmm_hessian"]

_FDTYPE = torch.float64


def gmm_reflectivity_torch(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                           free_surface: bool = False, solver: str = "riccati"):
    """Complex PP reflectivity (nfreq,) by the Global Matrix Method (``gmm_torch.py:229``).

    ``p`` may also be a 1-D tensor of slownesses, giving (n_p, nfreq).
    """
    if solver not in ("riccati", "dense"):
        raise ValueError(f"Unknown solver {solver!r}, expected 'riccati' or 'dense'")
    if not isinstance(omega, torch.Tensor):
        omega = torch.as_tensor(omega)
    dev = _device_for(alpha, omega)
    tab = D.table_from_tensors(alpha, beta, rho, thickness, Q_alpha, Q_beta, dev)
    p_t = torch.as_tensor(p, dtype=_FDTYPE).detach()
    R = D.gmm_reflectivity(tab, p_t.reshape(-1), omega.detach(), free_surface)
    R = R.to(omega.device)
    if p_t.dim() == 0:
        R = R[0]
    if _needs_grad(alpha, beta, rho, thickness):
        Rk = kennett_reflectivity_torch(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                                        free_surface)
        R = R + (Rk - Rk.detach())
    return R


def gmm_jacobian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p: float, omega,
                 free_surface: bool = False) -> torch.Tensor:
    """dR(omega_i)/dm_j over the packed parameters, shape (nfreq, 4N-1) (``gmm_torch.py:308``)."""
    return jacobian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                    free_surface=free_surface)


def gmm_hessian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p: float, omega, R_obs=None,
                free_surface: bool = False) -> torch.Tensor:
    """Hessian of ||R - R_obs||^2 over the packed parameters (``gmm_torch.py:340``)."""
    return hessian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, R_obs=R_obs,
                   free_surface=free_surface)
