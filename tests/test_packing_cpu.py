"""Parameter packing of the differentiable drop-ins (kennett_torch.py:552-608): the packed
vector m = [Vp_1..N, Vs_1..N, rho_1..N, h_1..N-1] (ocean and half-space thickness excluded,
4N - 1 values), its inverse, and the rows of the kernels' [4L] layer-parameter vector
(theta = alpha_l, beta_l, rho_l, h_l at k L + l) that form it."""

import numpy as np
import torch

from seismicinversion_b200.earth_models import random_layered_model
from seismicinversion_b200.kennett_torch import (_pack_params, _unpack_params, model_to_tensors,
                                                 packed_index)


def test_pack_unpack_and_index():
    m = random_layered_model(20, seed=2)
    t = model_to_tensors(m)
    L = m.n_layers
    packed = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"])
    assert packed.numel() == 4 * (L - 1) - 1 == 79
    a, b, r, h = _unpack_params(packed, t["alpha"], t["beta"], t["rho"], t["thickness"])
    for x, y in ((a, t["alpha"]), (b, t["beta"]), (r, t["rho"]), (h, t["thickness"])):
        assert torch.equal(x, y)
    full = torch.cat([t["alpha"], t["beta"], t["rho"], t["thickness"]])  # k L + l layout
    assert torch.equal(full[packed_index(L)], packed)
    # the half-space thickness is the torch path's 1e30 sentinel and stays out of m
    assert float(t["thickness"][-1]) == 1e30 and 1e30 not in packed.tolist()


def test_unpack_keeps_fixed_entries():
    m = random_layered_model(5, seed=4)
    t = model_to_tensors(m)
    packed = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"]) * 1.1
    a, b, r, h = _unpack_params(packed, t["alpha"], t["beta"], t["rho"], t["thickness"])
    assert a[0] == t["alpha"][0] and b[0] == t["beta"][0] and r[0] == t["rho"][0]
    assert h[0] == t["thickness"][0] and h[-1] == t["thickness"][-1]
    assert np.allclose(a[1:].numpy(), 1.1 * t["alpha"][1:].numpy())
