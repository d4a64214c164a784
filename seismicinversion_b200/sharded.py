"""Multi-GPU discrete-wavenumber gather: the slowness sum sharded over ranks.

One process per GPU (``torch.distributed``, NCCL over NVLink).  Rank k takes a contiguous
block of the slowness grid, computes its rows of R(p, omega + i gamma) and its partial
U(r, omega) = sum over its slownesses, then one all-reduce (sum) of U (n_r x n_omega complex,
3.3 MB for 100 offsets x 2047 frequencies) completes the sum on every rank, and each rank
forms the traces.  The R grid stays sharded (each rank holds its rows).  No other data
crosses ranks.  The reduction order differs from the single-GPU sum, so results agree to
rounding (~1e-16 relative).

The per-rank arithmetic is pluggable (``backend``): the default runs the library kernels on
the rank's GPU; tests substitute a CPU implementation to exercise the partitioning and the
collective on ``gloo`` ranks.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .earth_models import damped_gather_grid
from .layer_model import LayerModel
from .source import ricker_spectrum

__all__ = ["shard_range", "DeviceGatherBackend", "gather_sharded"]


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block [start, stop) of n items owned by ``rank`` of ``world`` (sizes differ
    by at most one; low ranks take the extra items)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class DeviceGatherBackend:
    """Per-rank arithmetic on the rank's GPU (library kernels)."""

    def __init__(self, device=None):
        from . import device as D

        self.D = D
        self.dev = D.require_cuda(device)

    def partial(self, model, p, pw, dp, omega_damped, omega_real, offsets, free_surface):
        D = self.D
        n_r, n_w = len(offsets), len(omega_real)
        if len(p) == 0:
            R = torch.empty((0, n_w), dtype=torch.complex128, device=self.dev)
            return R, torch.zeros((n_r, n_w), dtype=torch.complex128, device=self.dev)
        tab = D.layer_table(model, self.dev)
        R = D.reflectivity(tab, p, omega_damped, free_surface)
        return R, D.bessel_sum(R, p, pw, dp, omega_real, offsets)

    def traces(self, U, nw, S, decay):
        return self.D.traces(U, nw, S=S, decay=decay)


def gather_sharded(model: LayerModel, offsets, T: float = 64.0, nw: int = 2048,
                   np_slow: int = 4096, p_max: float = 1.2, gamma=None, source_func=None,
                   free_surface: bool = False, group=None, backend=None):
    """Gather with the slowness sum split over the ranks of ``group``.

    Same grid and result as ``compute_gather_gpu`` (``kennett_gather_gpu.py:169-284``).
    Returns ``(time, gather, R_shard, (p_start, p_stop))`` on every rank; ``gather`` and
    ``R_shard`` are tensors on the backend's device.
    """
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    backend = backend or DeviceGatherBackend()
    omega, omega_d, p, dp, taper, gamma = damped_gather_grid(T, nw, np_slow, p_max, gamma)
    wmax = nw * (2.0 * np.pi / T)
    S = ricker_spectrum(omega, wmax) if source_func is None else source_func(omega, wmax)
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    j0, j1 = shard_range(np_slow, rank, world)
    R, U = backend.partial(model, p[j0:j1], (taper * p)[j0:j1], dp, omega_d, omega,
                           np.asarray(offsets, dtype=np.float64), free_surface)
    dist.all_reduce(torch.view_as_real(U), op=dist.ReduceOp.SUM, group=group)
    g = backend.traces(U, nw, np.asarray(S, dtype=np.complex128), np.exp(-gamma * time))
    return time, g, R, (j0, j1)
