"""Drop-in for ``Kennett_Reflectivity.kennett_seismogram.compute_seismogram`` (``kennett_seismogram.py:57-150``)."""

from __future__ import annotations

import numpy as np

from . import device as _dev
from .earth_models import default_ocean_crust_model
from .layer_model import LayerModel
from .source import ricker_spectrum

__all__ = ["compute_seismogram", "default_ocean_crust_model"]


def compute_seismogram(model: LayerModel, p: float, T: float = 64.0, nw: int = 2048,
                       eps: float = 0.0, source_func=None, free_surface: bool = False):
    """``(time, seismogram)``: R at omega_k = k 2pi/T (k = 1..nw-1) times S, Hermitian FFT, x e^{eps t}."""
    dev = _dev.require_cuda()
    dw = 2.0 * np.pi / T
    omega = np.arange(1, nw, dtype=np.float64) * dw
    wmax = nw * dw
    S = ricker_spectrum(omega, wmax) if source_func is None else source_func(omega, wmax)
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    tab = _dev.layer_table(model, dev)
    R = _dev.reflectivity(tab, [float(p)], omega, free_surface)
    decay = None if eps == 0.0 else np.exp(eps * time)
    tr = _dev.traces(R, nw, S=np.asarray(S, dtype=np.complex128), decay=decay)
    return time, tr[0].cpu().numpy()
