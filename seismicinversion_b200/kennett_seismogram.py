"""Drop-in for ``Kennett_Reflectivity.kennett_seismogram.compute_seismogram`` (``kennett_seismogram.py:57-150``)."""

from __future__ import annotations

import numpy as np

from . import device as _dev
from .earth_models import default_ocean_crust_model
from .layer_model import LayerModel
from .source import ricker_spectrum

__all__ = ["compute_seismogram", "default_ocean_crust_model", "save_seismogram_txt"]


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


def save_seismogram_txt(path, time, seismogram) -> None:
    """Two columns (time, amplitude) as ``%.8e`` text -- the file the reference CLI writes
    (``kennett_seismogram.py:294-296``)."""
    np.savetxt(path, np.column_stack([time, seismogram]), fmt="%.8e")


def main(argv=None) -> None:
    """Command line as ``python -m Kennett_Reflectivity.kennett_seismogram``
    (``kennett_seismogram.py:153-296``): default 5-layer model, writes
    ``seismogram_p<p>.txt``.  Plotting is not provided."""
    import argparse

    ap = argparse.ArgumentParser(description="Synthetic seismogram via Kennett reflectivity (B200).")
    ap.add_argument("-p", "--slowness", type=float, default=0.2)
    ap.add_argument("-T", "--duration", type=float, default=64.0)
    ap.add_argument("-n", "--nw", type=int, default=2048)
    ap.add_argument("-o", "--output", default="seismogram_verification.png")
    ap.add_argument("--no-plot", action="store_true")
    ap.add_argument("--free-surface", action="store_true")
    args = ap.parse_args(argv)
    time, seis = compute_seismogram(default_ocean_crust_model(), args.slowness, T=args.duration,
                                    nw=args.nw, free_surface=args.free_surface)
    save_seismogram_txt(f"seismogram_p{args.slowness:.4f}.txt", time, seis)


if __name__ == "__main__":
    main()
