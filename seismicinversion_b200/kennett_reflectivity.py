"""Drop-in for ``Kennett_Reflectivity.kennett_reflectivity`` (``kennett_reflectivity.py:73-328``).

Same signature and result (complex128 R(omega) for one slowness), computed by the fused
sm_100a kernel.  ``omega`` may be real or complex (damped frequencies).  Torch CUDA tensors
are accepted and returned as tensors, keeping the data on the device.
"""

from __future__ import annotations

import numpy as np
import torch

from . import device as _dev
from .layer_model import LayerModel

__all__ = ["kennett_reflectivity", "inv2x2", "batch_inv2x2", "batch_matmul"]


def kennett_reflectivity(model: LayerModel, p: float, omega, free_surface: bool = False):
    """PP plane-wave reflectivity at slowness ``p`` for every frequency in ``omega``."""
    on_device = isinstance(omega, torch.Tensor) and omega.is_cuda
    dev = _dev.require_cuda(omega.device if on_device else None)
    tab = _dev.layer_table(model, dev)
    R = _dev.reflectivity(tab, [float(p)], omega, free_surface)[0]
    return R if on_device else R.cpu().numpy()


# Host-side 2x2 helpers exported by the reference package (kennett_reflectivity.py:18-70).
def inv2x2(M: np.ndarray) -> np.ndarray:
    a, b, c, d = M[0, 0], M[0, 1], M[1, 0], M[1, 1]
    return np.array([[d, -b], [-c, a]], dtype=M.dtype) / (a * d - b * c)


def batch_inv2x2(M: np.ndarray) -> np.ndarray:
    a, b, c, d = M[..., 0, 0], M[..., 0, 1], M[..., 1, 0], M[..., 1, 1]
    det = a * d - b * c
    out = np.empty_like(M)
    out[..., 0, 0] = d / det
    out[..., 0, 1] = -b / det
    out[..., 1, 0] = -c / det
    out[..., 1, 1] = a / det
    return out


def batch_matmul(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    if A.ndim in (2, 3) and B.ndim in (2, 3) and max(A.ndim, B.ndim) == 3:
        return np.matmul(A, B)
    raise ValueError(f"Unsupported shapes: {A.shape}, {B.shape}")
