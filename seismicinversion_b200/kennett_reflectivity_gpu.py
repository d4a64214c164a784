"""Drop-in for ``Kennett_Reflectivity.kennett_reflectivity_gpu`` (``kennett_reflectivity_gpu.py:39-275``).

``kennett_reflectivity_batch`` computes the whole (slowness x frequency) grid in one launch
of the fused kernel (the reference runs batched NumPy on the CPU).  ``get_device`` returns
the CUDA device; there is no MPS/CPU alternative.
"""

from __future__ import annotations

import torch

from . import device as _dev
from .layer_model import LayerModel

__all__ = ["kennett_reflectivity_batch", "get_device"]


def get_device() -> torch.device:
    """The CUDA device the kernels run on (raises if none: no CPU fallback)."""
    return _dev.require_cuda()


def kennett_reflectivity_batch(model: LayerModel, p_samples, omega, free_surface: bool = False):
    """R of shape ``(np_slow, nfreq)`` complex128 for all slownesses at once.

    NumPy in -> NumPy out (as the reference); CUDA tensors in -> CUDA tensor out.
    """
    on_device = isinstance(omega, torch.Tensor) and omega.is_cuda
    dev = _dev.require_cuda(omega.device if on_device else None)
    tab = _dev.layer_table(model, dev)
    R = _dev.reflectivity(tab, p_samples, omega, free_surface)
    return R if on_device else R.cpu().numpy()
