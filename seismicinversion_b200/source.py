"""Source wavelets (``Kennett_Reflectivity/source.py``).

The spectrum is evaluated on the host in float64 (nw values, negligible cost) and uploaded,
so the device multiplies by exactly the numbers the reference uses.
"""

from __future__ import annotations

import numpy as np

__all__ = ["ricker_spectrum", "ricker_wavelet", "ricker_10hz"]


def ricker_spectrum(omega: np.ndarray, omega_max: float) -> np.ndarray:
    """S = Z exp(-Z + i omega T0), Z = omega^2 / (4 a^2), a = 0.1 omega_max, T0 = 5 / (a sqrt 2).

    Same parameterisation as ``source.py:10-45``: |S| peaks at omega = 2a = 0.2 omega_max.
    """
    a = 0.1 * omega_max
    t0 = 5.0 / (a * np.sqrt(2.0))
    z = (omega**2) / (4.0 * a**2)
    return z * np.exp(-z + 1j * omega * t0)


def ricker_wavelet(t: np.ndarray, f_peak: float) -> np.ndarray:
    """Time-domain Ricker wavelet (``source.py:48-80``)."""
    t0 = 1.0 / (np.pi * f_peak)
    tau = np.pi * f_peak * (t - t0)
    return (1.0 - 2.0 * tau**2) * np.exp(-(tau**2))


def ricker_10hz(omega: np.ndarray, omega_max: float) -> np.ndarray:
    """Ricker spectrum peaking at 10 Hz: ``ricker_spectrum(omega, 100 pi)`` (omega_max is ignored).

    The reference parameterises its Ricker by ``omega_max`` (peak at 0.2 omega_max); passing
    this through the ``source_func`` hook gives a 10 Hz peak at any T / nw.
    """
    return ricker_spectrum(omega, 100.0 * np.pi)
