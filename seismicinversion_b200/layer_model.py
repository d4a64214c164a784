"""Plane-layered earth model: the host-side description handed to the GPU kernels.

Mirrors the reference's ``LayerModel`` (``Kennett_Reflectivity/layer_model.py:77-167``):
structure-of-arrays float64 ``alpha, beta, rho, thickness, Q_alpha, Q_beta`` with the same
validation and the same ``ValueError`` messages, so code written against the reference keeps
working.  ``complex_slowness`` / ``vertical_slowness`` are the scalar host versions
(``layer_model.py:15-45`` and ``:48-74``); the kernels evaluate the same formulas on the
device.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = [
    "LayerModel",
    "complex_slowness",
    "vertical_slowness",
    "pack_layers",
    "HALF_SPACE_SENTINEL",
]

#: Thicknesses at or above this value (and +inf) are treated as the half-space: its phase
#: factors are exactly 1.  This accepts both the NumPy convention (``np.inf``,
#: ``kennett_reflectivity.py:179``) and the torch convention (``1e30`` sentinel,
#: ``kennett_torch.py:374-375``, ``:709-710``).
HALF_SPACE_SENTINEL = 1e30


def complex_slowness(velocity: float, Q: float) -> complex:
    """Attenuating slowness s = (4Q^2 + 2iQ) / ((1 + 4Q^2) v).

    Same formula and argument checks as ``layer_model.py:15-45``.
    """
    if velocity <= 0:
        raise ValueError(f"velocity must be positive, got {velocity}")
    if Q <= 0:
        raise ValueError(f"Q must be positive, got {Q}")
    q2 = 2.0 * Q
    q2sq = q2 * q2
    den = (1.0 + q2sq) * velocity
    return complex(q2sq / den, q2 / den)


def vertical_slowness(slowness: complex, p: complex) -> complex:
    """eta = sqrt((s + p)(s - p)) on the branch with Im(eta) > 0 (``layer_model.py:48-74``)."""
    t = (slowness + p) * (slowness - p)
    eta = complex(np.sqrt(complex(t)))
    if eta.imag <= 0.0:
        eta = -eta
    return eta


@dataclass
class LayerModel:
    """Stratified elastic model: layer 0 is the acoustic ocean, the last layer the half-space."""

    alpha: np.ndarray
    beta: np.ndarray
    rho: np.ndarray
    thickness: np.ndarray
    Q_alpha: np.ndarray
    Q_beta: np.ndarray

    def __post_init__(self) -> None:
        for name in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta"):
            setattr(self, name, np.asarray(getattr(self, name), dtype=np.float64))
        n = self.n_layers
        for name in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta"):
            if len(getattr(self, name)) != n:
                raise ValueError(f"{name} length mismatch: expected {n}")
        if np.any(self.alpha <= 0):
            raise ValueError("All alpha must be positive")
        if np.any(self.beta < 0):
            raise ValueError("All beta must be non-negative")
        if np.any(self.rho <= 0):
            raise ValueError("All rho must be positive")

    @property
    def n_layers(self) -> int:
        return len(self.alpha)

    @classmethod
    def from_arrays(cls, alpha, beta, rho, thickness, Q_alpha, Q_beta) -> "LayerModel":
        return cls(alpha, beta, rho, thickness, Q_alpha, Q_beta)

    def complex_slowness_p(self) -> np.ndarray:
        return np.array(
            [complex_slowness(a, q) for a, q in zip(self.alpha, self.Q_alpha)],
            dtype=np.complex128,
        )

    def complex_slowness_s(self) -> np.ndarray:
        out = np.zeros(self.n_layers, dtype=np.complex128)
        for i in range(self.n_layers):
            if self.beta[i] > 0:
                out[i] = complex_slowness(self.beta[i], self.Q_beta[i])
        return out

    def complex_velocity_s(self) -> np.ndarray:
        ss = self.complex_slowness_s()
        out = np.zeros(self.n_layers, dtype=np.complex128)
        nz = np.abs(ss) > 0
        out[nz] = 1.0 / ss[nz]
        return out


def pack_layers(model: LayerModel) -> np.ndarray:
    """Pack a model into the kernels' layer table: float64 ``[6, n_layers]``.

    Rows are alpha, beta, rho, thickness, Q_alpha, Q_beta.  ``+inf`` thicknesses are kept
    (the device treats ``inf`` and values >= 1e30 as the half-space).

    Beyond the reference's own checks this rejects what the kernels cannot evaluate:
    fewer than two layers, a non-acoustic top layer (the ocean-bottom coefficients assume
    beta_0 = 0, ``scattering_matrices.py:164-296``), non-finite or non-positive Q, negative
    or NaN thickness.
    """
    n = model.n_layers
    if n < 2:
        raise ValueError(f"model needs at least 2 layers (ocean + half-space), got {n}")
    if model.beta[0] != 0.0:
        raise ValueError(f"layer 0 must be the acoustic ocean (beta=0), got beta={model.beta[0]}")
    tab = np.empty((6, n), dtype=np.float64)
    tab[0] = model.alpha
    tab[1] = model.beta
    tab[2] = model.rho
    tab[3] = model.thickness
    tab[4] = model.Q_alpha
    tab[5] = model.Q_beta
    if not np.all(np.isfinite(tab[[0, 1, 2, 4, 5]])):
        raise ValueError("alpha, beta, rho, Q_alpha and Q_beta must be finite")
    if np.any(model.Q_alpha <= 0) or np.any(model.Q_beta[model.beta > 0] <= 0):
        raise ValueError("Q_alpha (all layers) and Q_beta (elastic layers) must be positive")
    if np.any(np.isnan(model.thickness)) or np.any(model.thickness < 0):
        raise ValueError("thickness must be non-negative (inf or >= 1e30 for the half-space)")
    return tab


def is_half_space(h: float) -> bool:
    return math.isinf(h) or h >= HALF_SPACE_SENTINEL
