"""Training data for amortized inference, generated with the batched forward kernels.

Mirror of ``NeuralInversion/inference_data.py`` (``generate_training_data`` :72-176,
``_perturb_model`` :37-69, ``ReflectivityDataset`` :179-210): the same prior (uniform
multiplicative perturbations of a reference model's packed sub-ocean parameters, drawn with
the same generator calls in the same order, so a seed gives the same parameter samples), the
same frequency grid (omega_k = k 2pi/64, k = 1..nfreq) and the same ``.pt`` file layout
(float32 ``log_params`` and ``reflectivity`` = [Re R | Im R] per slowness).  The forward
model is the Kennett kernel; the reference computes it with its global-matrix (Riccati)
solver, which agrees with Kennett to < 1e-10 (``GlobalMatrix/test_gmm.py:25-51``), far
below the float32 storage precision.  Samples are evaluated in chunks of ``chunk`` models,
each chunk one persistent batched launch.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from . import device as D
from .batch import ModelBatch
from .earth_models import default_ocean_crust_model
from .layer_model import LayerModel, pack_layers

__all__ = ["DataGenConfig", "generate_training_data", "ReflectivityDataset", "perturb_model"]


@dataclass
class DataGenConfig:
    """Data-generation settings (``NeuralInversion/inference_config.py:31-57``)."""

    n_train: int = 50_000
    n_val: int = 5_000
    n_test: int = 5_000
    velocity_perturbation: float = 0.20
    density_perturbation: float = 0.15
    thickness_perturbation: float = 0.25
    p_values: list = field(default_factory=lambda: [0.05, 0.10, 0.15, 0.20, 0.25, 0.30,
                                                     0.35, 0.40, 0.45, 0.50, 0.55, 0.60])
    nfreq: int = 64
    seed: int = 42


def perturb_model(true_params: np.ndarray, n_sub: int, rng: np.random.Generator,
                  vel_pert: float, den_pert: float, thick_pert: float) -> np.ndarray:
    """One prior sample: uniform factors on velocities, densities, thicknesses (in that order)."""
    n = len(true_params)
    f = np.ones(n)
    n_vel, n_thick = 2 * n_sub, n_sub - 1
    f[:n_vel] = rng.uniform(1.0 - vel_pert, 1.0 + vel_pert, n_vel)
    f[n_vel:n_vel + n_sub] = rng.uniform(1.0 - den_pert, 1.0 + den_pert, n_sub)
    f[n_vel + n_sub:n_vel + n_sub + n_thick] = rng.uniform(1.0 - thick_pert, 1.0 + thick_pert,
                                                           n_thick)
    return true_params * f


def _tables(ref: LayerModel, params: np.ndarray) -> np.ndarray:
    """Layer tables [n, 6, L] for packed sub-ocean parameter rows (ocean and half-space
    thickness fixed to the reference's)."""
    tab0 = pack_layers(ref)
    L = ref.n_layers
    n_sub = L - 1
    n = params.shape[0]
    tabs = np.repeat(tab0[None], n, axis=0)
    tabs[:, 0, 1:] = params[:, :n_sub]
    tabs[:, 1, 1:] = params[:, n_sub:2 * n_sub]
    tabs[:, 2, 1:] = params[:, 2 * n_sub:3 * n_sub]
    tabs[:, 3, 1:L - 1] = params[:, 3 * n_sub:]
    return tabs


def generate_training_data(output_dir, config: DataGenConfig | None = None,
                           ref_model: LayerModel | None = None, chunk: int = 16384,
                           device=None) -> dict:
    """Generate train / val / test ``.pt`` files; returns {split: path}."""
    config = config or DataGenConfig()
    ref = ref_model or default_ocean_crust_model()
    dev = D.require_cuda(device)
    out = Path(output_dir)
    out.mkdir(parents=True, exist_ok=True)
    L = ref.n_layers
    n_sub = L - 1
    true = np.concatenate([ref.alpha[1:], ref.beta[1:], ref.rho[1:], ref.thickness[1:-1]])
    n_params = len(true)
    p = np.asarray(config.p_values, dtype=np.float64)
    omega = np.arange(1, config.nfreq + 1, dtype=np.float64) * (2.0 * np.pi / 64.0)
    rng = np.random.default_rng(config.seed)
    paths = {}
    for split, n in (("train", config.n_train), ("val", config.n_val), ("test", config.n_test)):
        params = np.empty((n, n_params))
        for i in range(n):
            params[i] = perturb_model(true, n_sub, rng, config.velocity_perturbation,
                                      config.density_perturbation,
                                      config.thickness_perturbation)
        refl = torch.empty((n, len(p), 2 * config.nfreq), dtype=torch.float32)
        for c0 in range(0, n, chunk):
            tabs = _tables(ref, params[c0:c0 + chunk])
            batch = ModelBatch.from_tables(tabs, p, omega, device=dev)
            batch.launch()
            R = batch.R[:tabs.shape[0] * len(p) * len(omega)].view(tabs.shape[0], len(p), len(omega))
            x = torch.cat([R.real, R.imag], dim=-1).float()
            refl[c0:c0 + tabs.shape[0]] = x.cpu()
        path = out / f"{split}.pt"
        torch.save({"log_params": torch.tensor(np.log(params), dtype=torch.float32),
                    "reflectivity": refl, "p_values": list(config.p_values),
                    "nfreq": config.nfreq, "n_params": n_params}, path)
        paths[split] = path
    return paths


class ReflectivityDataset(torch.utils.data.Dataset):
    """(reflectivity (n_p, 2 nfreq) float32, log_params) pairs from a generated file,
    optionally scaled by the sample's max |x| (``inference_data.py:179-210``)."""

    def __init__(self, path, normalise: bool = True) -> None:
        data = torch.load(path, weights_only=True)
        self.reflectivity = data["reflectivity"]
        self.log_params = data["log_params"]
        self.p_values = data["p_values"]
        self.nfreq = data["nfreq"]
        self.normalise = normalise

    def __len__(self) -> int:
        return len(self.log_params)

    def __getitem__(self, idx):
        x = self.reflectivity[idx]
        if self.normalise:
            x = x / x.abs().max().clamp(min=1e-10)
        return x, self.log_params[idx]
