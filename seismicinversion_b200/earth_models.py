"""Seeded synthetic earth models and grids for the benchmark workloads.

The reference ships no datasets; every workload is synthetic.  Models are drawn as:
1 km water layer (Vp 1.5 km/s, Vs 0, rho 1.0 g/cc) over ``n_sub`` sub-ocean layers whose
last one is the half-space; sub-ocean Vp ~ sort(U(1.8, 5.0)) increasing with depth,
Vs = Vp / U(1.7, 2.0), rho = 0.31 (1000 Vp)^0.25, h ~ U(0.2, 1.0) km, half-space h = inf,
Q_alpha = 100 and Q_beta = 50 in every layer.  Draw order is fixed (Vp, Vs ratio, h) so a
seed names a model exactly.
"""

from __future__ import annotations

import numpy as np

from .layer_model import LayerModel

__all__ = [
    "random_layered_model",
    "default_ocean_crust_model",
    "seismogram_omega",
    "damped_gather_grid",
    "uneven_batch_specs",
]


def random_layered_model(n_sub: int, seed: int, water_depth: float = 1.0) -> LayerModel:
    """Water layer over ``n_sub`` random sub-ocean layers (the last is the half-space).

    ``n_sub = 5`` gives the 6-layer single-trace model, ``n_sub = 20`` the 21-layer
    (79-parameter) gather / inversion model.
    """
    if n_sub < 1:
        raise ValueError("n_sub must be >= 1")
    rng = np.random.default_rng(seed)
    vp = np.sort(rng.uniform(1.8, 5.0, n_sub))
    vs = vp / rng.uniform(1.7, 2.0, n_sub)
    rho = 0.31 * (1000.0 * vp) ** 0.25
    h = rng.uniform(0.2, 1.0, n_sub)
    h[-1] = np.inf
    return LayerModel.from_arrays(
        alpha=np.concatenate([[1.5], vp]),
        beta=np.concatenate([[0.0], vs]),
        rho=np.concatenate([[1.0], rho]),
        thickness=np.concatenate([[water_depth], h]),
        Q_alpha=np.full(n_sub + 1, 100.0),
        Q_beta=np.full(n_sub + 1, 50.0),
    )


def default_ocean_crust_model() -> LayerModel:
    """The reference's 5-layer default model (``kennett_seismogram.py:25-54``)."""
    return LayerModel.from_arrays(
        alpha=[1.5, 1.6, 3.0, 5.0, 2.2],
        beta=[0.0, 0.3, 1.5, 3.0, 1.1],
        rho=[1.0, 2.0, 3.0, 3.0, 1.8],
        thickness=[2.0, 1.0, 1.0, 1.0, np.inf],
        Q_alpha=[20000, 100, 100, 100, 100],
        Q_beta=[1e10, 100, 100, 100, 100],
    )


def seismogram_omega(T: float = 64.0, nw: int = 2048) -> np.ndarray:
    """omega_k = k * 2 pi / T, k = 1..nw-1 (DC and Nyquist dropped, ``kennett_seismogram.py:104-110``)."""
    dw = 2.0 * np.pi / T
    return np.arange(1, nw, dtype=np.float64) * dw


def damped_gather_grid(T: float, nw: int, np_slow: int, p_max: float, gamma: float | None = None):
    """Frequency and slowness grids of the discrete-wavenumber gather (``kennett_gather.py:198-225``).

    Returns ``(omega_real, omega_damped, p_samples, dp, taper, gamma)``.
    """
    if gamma is None:
        gamma = np.pi / T
    omega = seismogram_omega(T, nw)
    dp = p_max / np_slow
    p = np.arange(1, np_slow + 1, dtype=np.float64) * dp
    taper = 0.5 * (1.0 + np.cos(np.pi * p / p_max))
    return omega, omega + 1j * gamma, p, dp, taper, gamma


def uneven_batch_specs(n_models: int, seed: int, n_layers_range=(3, 64),
                       nw_choices=(256, 512, 1024, 2048), np_range=(16, 256), p_max: float = 0.8):
    """Model / grid specs of the uneven-batching workload.

    Each entry: ``(model, p_samples, omega)`` with total layers ~ U{3..64} (water + sub-ocean),
    n_omega from ``nw_choices`` with omega_k = k 2 pi / 64 (k = 1..n_omega) and
    n_p ~ U{16..256} with p_j = j p_max / n_p.
    """
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_models):
        L = int(rng.integers(n_layers_range[0], n_layers_range[1] + 1))
        nw = int(rng.choice(nw_choices))
        npp = int(rng.integers(np_range[0], np_range[1] + 1))
        model = random_layered_model(L - 1, seed=int(rng.integers(0, 2**31 - 1)))
        omega = np.arange(1, nw + 1, dtype=np.float64) * (2.0 * np.pi / 64.0)
        p = np.arange(1, npp + 1, dtype=np.float64) * (p_max / npp)
        specs.append((model, p, omega))
    return specs
