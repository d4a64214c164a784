"""Drop-in for ``Kennett_Reflectivity.kennett_gather.compute_gather`` (``kennett_gather.py:127-305``).

Same signature and defaults (np_slow = 2048, p_max = 1.0); computed on the GPU by the same
path as ``compute_gather_gpu``.  ``n_workers`` is accepted for compatibility and ignored (the
reference's process pool has no counterpart: the slowness loop is a kernel grid axis).
"""

from __future__ import annotations

import numpy as np

from .earth_models import default_ocean_crust_model
from .kennett_gather_gpu import gather_device
from .layer_model import LayerModel

__all__ = ["compute_gather", "default_ocean_crust_model"]


def compute_gather(model: LayerModel, offsets, T: float = 64.0, nw: int = 2048,
                   np_slow: int = 2048, p_max: float = 1.0, gamma=None, source_func=None,
                   n_workers=None, free_surface: bool = False):
    time, _, _, g = gather_device(model, offsets, T, nw, np_slow, p_max, gamma, source_func,
                                  free_surface)
    return time, np.asarray(offsets), g.cpu().numpy()
