"""Amortized-inference training data on the batched kernels vs the reference generator
(golden file from NeuralInversion.generate_training_data, GMM forward): identical parameter
samples (same prior draws) and reflectivity equal to float32 storage precision."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_matches_reference_generator(golden, tmp_path):
    from seismicinversion_b200.training_data import DataGenConfig, ReflectivityDataset, generate_training_data

    g = golden("training_data_small.npz")
    cfg = DataGenConfig(n_train=12, n_val=4, n_test=4, nfreq=32, seed=42)
    paths = generate_training_data(tmp_path, cfg, chunk=5)
    for split in ("train", "val", "test"):
        data = torch.load(paths[split], weights_only=True)
        assert np.array_equal(data["log_params"].numpy(), g[f"{split}_log_params"])
        x, ref = data["reflectivity"].numpy(), g[f"{split}_reflectivity"]
        assert x.shape == ref.shape and x.dtype == np.float32
        assert np.max(np.abs(x - ref)) <= 4e-7 * np.max(np.abs(ref))
    ds = ReflectivityDataset(paths["train"])
    xb, yb = ds[3]
    assert xb.shape == (12, 64) and float(xb.abs().max()) == pytest.approx(1.0)
