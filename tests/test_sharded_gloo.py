"""Multi-rank gather on CPU: two gloo ranks split the slowness sum, all-reduce U, and must
reproduce the single-process oracle gather (1e-12).  The per-rank arithmetic is the oracle
(test-only backend), so this checks the partitioning and the collective, not the kernels."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from seismicinversion_b200.sharded import shard_range


def test_shard_range_partitions():
    for n in (0, 1, 7, 8192, 8193):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


class OracleBackend:
    def partial(self, model, p, pw, dp, omega_damped, omega_real, offsets, free_surface):
        from oracle import kennett_oracle as O

        m = model
        n_r, n_w = len(offsets), len(omega_real)
        if len(p) == 0:
            return (torch.zeros((0, n_w), dtype=torch.complex128),
                    torch.zeros((n_r, n_w), dtype=torch.complex128))
        R = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p,
                           omega_damped, free_surface)
        U = O.bessel_sum(R, p, omega_real, offsets, dp, taper=pw / p)
        return torch.as_tensor(R), torch.as_tensor(U)

    def traces(self, U, nw, S, decay):
        from oracle import kennett_oracle as O

        return torch.as_tensor(O.hermitian_traces(U.numpy() * S, nw, decay))


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from seismicinversion_b200.earth_models import random_layered_model
        from seismicinversion_b200.sharded import gather_sharded

        m = random_layered_model(6, seed=31)
        offs = np.array([1.0, 4.0, 9.0])
        _, g, R, span = gather_sharded(m, offs, T=32.0, nw=64, np_slow=37, p_max=1.0,
                                       free_surface=True, backend=OracleBackend())
        out[rank] = (g.numpy(), R.numpy(), span)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_single_process():
    from oracle import kennett_oracle as O
    from seismicinversion_b200.earth_models import random_layered_model

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    m = random_layered_model(6, seed=31)
    _, _, g_ref, R_ref = O.gather(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta,
                                  np.array([1.0, 4.0, 9.0]), T=32.0, nw=64, np_slow=37,
                                  p_max=1.0, free_surface=True)
    spans = [out[r][2] for r in range(2)]
    assert spans == [(0, 19), (19, 37)]
    for r in range(2):
        g, R, (a, b) = out[r]
        scale = np.max(np.abs(g_ref))
        assert np.max(np.abs(g - g_ref)) / scale < 1e-12
        assert np.max(np.abs(R - R_ref[a:b])) / np.max(np.abs(R_ref)) < 1e-13
