"""Stream capture of the launch entry points: after one eager call per size (which raises the
kernels' shared-memory limits and creates the cuFFT plan), the forward (a 130-layer model,
whose block needs more than 48 KB of shared memory), GMM, Bessel-sum, traces and misfit-
gradient calls record into one CUDA graph under torch's default (global) capture mode, and
its replay equals the eager results bit for bit."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_entry_points_capture_into_a_graph():
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    dev = torch.device("cuda:0")
    big = D.layer_table(random_layered_model(129, seed=41), dev)
    small = D.layer_table(random_layered_model(8, seed=42), dev)
    n_p, n_w = 96, 300
    p = torch.as_tensor(np.arange(1, n_p + 1) * (1.0 / n_p), device=dev)
    om = torch.as_tensor(np.arange(1, n_w + 1) * (2 * np.pi / 64), device=dev)
    w = (om + 1j * (np.pi / 64)).to(torch.complex128)
    pw = 0.5 * (1.0 + torch.cos(np.pi * p)) * p
    offs = torch.as_tensor([0.5, 3.0, 11.0, 27.5], device=dev)
    S = torch.ones(n_w, dtype=torch.complex128, device=dev)
    decay = torch.ones(2 * (n_w + 1), dtype=torch.float64, device=dev)
    R_obs = 0.9 * D.reflectivity(small, p, w, True)

    def run():
        Rb = D.reflectivity(big, p, w, True)
        Rg = D.gmm_reflectivity(small, p, w, True)
        U = D.bessel_sum(Rg, p, pw, 1.0 / n_p, om, offs)
        g = D.traces(U, n_w + 1, S=S, decay=decay)
        cg, _ = D.misfit_gradient(small, p, w, R_obs, True)
        return Rb, Rg, U, g, cg

    eager = [x.clone() for x in run()]
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        static = run()
    for _ in range(2):
        graph.replay()
        torch.cuda.synchronize()
        for a, b in zip(static, eager):
            assert torch.equal(a, b)
