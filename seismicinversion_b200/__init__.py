"""seismicinversion_b200 -- B200-native (sm_100a, FP64) Kennett reflectivity path.

A drop-in for the hot path of tmnestor/SeismicInversion's ``Kennett_Reflectivity``
package: ``kennett_reflectivity``, ``kennett_reflectivity_batch``, ``compute_gather_gpu`` /
``compute_gather``, ``compute_seismogram`` and the differentiable
``kennett_reflectivity_torch`` used by the tau-p inversion.  Names resolve lazily, as in the
reference's ``__init__`` (``Kennett_Reflectivity/__init__.py:70-179``).  Every compute entry
point runs in ``libkennett_b200.so``; there is no CPU fallback.
"""

from __future__ import annotations

from .kennett_reflectivity import batch_inv2x2, batch_matmul, inv2x2, kennett_reflectivity
from .layer_model import LayerModel, complex_slowness, vertical_slowness
from .source import ricker_spectrum, ricker_wavelet

__version__ = "1.0.0"

_LAZY = {
    "compute_seismogram": ".kennett_seismogram",
    "default_ocean_crust_model": ".earth_models",
    "compute_gather": ".kennett_gather",
    "compute_gather_gpu": ".kennett_gather_gpu",
    "kennett_reflectivity_batch": ".kennett_reflectivity_gpu",
    "get_device": ".kennett_reflectivity_gpu",
    "kennett_reflectivity_torch": ".kennett_torch",
    "forward_model_torch": ".kennett_torch",
    "jacobian": ".kennett_torch",
    "hessian": ".kennett_torch",
    "model_to_tensors": ".kennett_torch",
    "InversionResult": ".taup_inversion",
    "compute_taup_traces": ".taup_inversion",
    "invert_taup": ".taup_inversion",
    "taup_misfit_grad_hessian": ".taup_inversion",
    "invert_taup_batch": ".taup_batch",
    "gmm_reflectivity": ".global_matrix",
    "gmm_reflectivity_torch": ".gmm_torch",
    "gmm_jacobian": ".gmm_torch",
    "gmm_hessian": ".gmm_torch",
}

__all__ = ["LayerModel", "complex_slowness", "vertical_slowness", "ricker_spectrum",
           "ricker_wavelet", "kennett_reflectivity", "inv2x2", "batch_inv2x2", "batch_matmul",
           *_LAZY]


def __getattr__(name: str):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    import importlib

    return getattr(importlib.import_module(mod, __name__), name)
