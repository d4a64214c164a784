"""Drop-in for ``GlobalMatrix.global_matrix.gmm_reflectivity`` (``global_matrix.py:297-348``).

Same signature and result (complex128 R(omega) for one slowness by the Global Matrix Method),
computed by the block-Riccati kernel ``kr_gmm_reflectivity``: an FP64 evaluation of the
reflectivity independent of the Kennett recursion (4x4 continuity systems per interface
instead of 2x2 reflection/transmission matrices).  ``solver="dense"`` (the reference's
O(N^3) full-system solve) is accepted and answered by the same O(N) Riccati kernel, whose
result the reference's own tests hold equal to the dense solve to 1e-10
(``GlobalMatrix/test_riccati.py:57-79``).
"""

from __future__ import annotations

import torch

from . import device as _dev
from .layer_model import LayerModel

__all__ = ["gmm_reflectivity"]


def gmm_reflectivity(model: LayerModel, p: float, omega, free_surface: bool = False,
                     solver: str = "riccati"):
    """PP plane-wave reflectivity at slowness ``p`` for every frequency in ``omega``."""
    if solver not in ("riccati", "dense"):
        raise ValueError(f"Unknown solver {solver!r}, expected 'riccati' or 'dense'")
    on_device = isinstance(omega, torch.Tensor) and omega.is_cuda
    dev = _dev.require_cuda(omega.device if on_device else None)
    tab = _dev.layer_table(model, dev)
    R = _dev.gmm_reflectivity(tab, [float(p)], omega, free_surface)[0]
    return R if on_device else R.cpu().numpy()
