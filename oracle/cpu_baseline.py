"""CPU baseline of the gather workload -- TEST / BENCH INFRASTRUCTURE ONLY.

Times the oracle (the NumPy/SciPy restatement of the reference, pinned to the reference's
golden vectors) on the host cores, organised the way the reference's CPU gather runs it:
a ``multiprocessing`` pool over slowness batches, each worker computing R(omega + i gamma)
for its slownesses and their J0-weighted contribution to U(r, omega)
(``kennett_gather.py:57-124``, ``:246-288``).  Used by ``bench.py`` for its ``cpu_baseline``
and ``--impl reference`` legs.  Pools are created with the ``spawn`` start method.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np

from . import kennett_oracle as O


def _init_worker():
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["MKL_NUM_THREADS"] = "1"


def _work(args):
    (layers, p, omega_damped, offsets, pw, dp, fs) = args
    alpha, beta, rho, h, qa, qb = layers
    R = O.reflectivity(alpha, beta, rho, h, qa, qb, p, omega_damped, fs)
    U = O.bessel_sum(R, p, omega_damped.real, offsets, dp, taper=pw / p)
    return R, U


class GatherBaseline:
    """Bounded-sample timing of the CPU gather on ``workers`` processes."""

    def __init__(self, model, offsets, T, nw, np_slow, p_max, free_surface, n_sample,
                 workers=None, chunk=2):
        self.workers = workers or len(os.sched_getaffinity(0))
        self.layers = tuple(np.asarray(getattr(model, k), dtype=np.float64) for k in
                            ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta"))
        self.offsets = np.asarray(offsets, dtype=np.float64)
        gamma = np.pi / T
        dw = 2.0 * np.pi / T
        self.omega_damped = np.arange(1, nw, dtype=np.float64) * dw + 1j * gamma
        dp = p_max / np_slow
        p_all = np.arange(1, np_slow + 1, dtype=np.float64) * dp
        taper = 0.5 * (1.0 + np.cos(np.pi * p_all / p_max))
        n_sample = min(n_sample, np_slow)
        self.rows = np.unique(np.linspace(0, np_slow - 1, n_sample).round().astype(int))
        self.p = p_all[self.rows]
        self.pw = (taper * p_all)[self.rows]
        self.dp = dp
        self.fs = free_surface
        self.chunk = chunk
        self.n_layers = len(self.layers[0])
        ctx = mp.get_context("spawn")
        self.pool = ctx.Pool(self.workers, initializer=_init_worker)

    def tasks(self):
        out = []
        for k in range(0, len(self.p), self.chunk):
            sl = slice(k, k + self.chunk)
            out.append((self.layers, self.p[sl], self.omega_damped, self.offsets, self.pw[sl],
                        self.dp, self.fs))
        return out

    def warm(self):
        """Start every worker (spawn, imports) on a small task before a timed step."""
        t = self.tasks()[:1]
        self.pool.map(_work, t * self.workers, chunksize=1)

    def step(self):
        """One timed sample: returns (seconds, R rows (n_sample, nw-1), U partial)."""
        t0 = time.perf_counter()
        res = self.pool.map(_work, self.tasks(), chunksize=1)
        dt = time.perf_counter() - t0
        R = np.concatenate([r for r, _ in res], axis=0)
        U = sum(u for _, u in res)
        return dt, R, U

    def updates(self):
        """(omega, p, interface) updates in one sample."""
        return len(self.p) * len(self.omega_damped) * (self.n_layers - 1)

    def close(self):
        self.pool.close()
        self.pool.join()


def _warm(_):
    import torch  # noqa: F401

    from . import torch_oracle  # noqa: F401
    return 0


def _refl_chunk(args):
    layers, p, omega, fs = args
    return O.reflectivity(*layers, p, omega, fs)


def _grad_chunk(args):
    """chi and its gradient d chi / d(alpha, beta, rho, h) [4L] on a slowness subset, by
    torch autograd through the differentiable oracle (one thread per worker)."""
    import torch

    from . import torch_oracle as T

    torch.set_num_threads(1)
    layers, p, omega, R_obs, fs = args
    t = [torch.as_tensor(np.asarray(x, dtype=np.float64)) for x in layers]
    for x in t[:4]:
        x.requires_grad_(True)
    R = T.reflectivity(*t, p, torch.as_tensor(omega), fs)
    chi = T.misfit(R, torch.as_tensor(np.asarray(R_obs)))
    g = torch.autograd.grad(chi, t[:4])
    return float(chi.detach()), np.concatenate([x.numpy() for x in g])


def _layers(model):
    return tuple(np.asarray(getattr(model, k), dtype=np.float64) for k in
                 ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta"))


class ReflectivityPool:
    """The oracle's reflectivity (and misfit gradient) over a slowness grid, split into
    slowness chunks across a ``spawn`` process pool (test infrastructure: full-size parity
    checks of the batched and served paths, and CPU baselines of those workloads)."""

    def __init__(self, workers=None):
        self.workers = workers or len(os.sched_getaffinity(0))
        self.pool = mp.get_context("spawn").Pool(self.workers, initializer=_init_worker)

    def reflectivity(self, model, p, omega, free_surface=False):
        layers = _layers(model)
        p = np.asarray(p, dtype=np.float64)
        omega = np.asarray(omega, dtype=np.complex128)
        n = max(1, min(len(p), 2 * self.workers))
        chunks = [c for c in np.array_split(p, n) if len(c)]
        res = self.pool.map(_refl_chunk, [(layers, c, omega, free_surface) for c in chunks],
                            chunksize=1)
        return np.concatenate(res, axis=0)

    def misfit_gradient(self, model, p, omega, R_obs, free_surface=False):
        """(chi, gradient [4L]) of chi = sum |R - R_obs|^2, the slowness sum split across the
        workers (torch autograd through the differentiable oracle)."""
        layers = _layers(model)
        p = np.asarray(p, dtype=np.float64)
        R_obs = np.asarray(R_obs, dtype=np.complex128).reshape(len(p), -1)
        n = max(1, min(len(p), 2 * self.workers))
        idx = [c for c in np.array_split(np.arange(len(p)), n) if len(c)]
        res = self.pool.map(_grad_chunk, [(layers, p[c], omega, R_obs[c], free_surface)
                                          for c in idx], chunksize=1)
        return sum(r[0] for r in res), sum(r[1] for r in res)

    def timed_jobs(self, fn, jobs):
        """Seconds to run ``jobs`` (argument tuples of ``fn``) across the pool."""
        t0 = time.perf_counter()
        self.pool.map(fn, jobs, chunksize=1)
        return time.perf_counter() - t0

    def warm(self):
        """Start every worker (spawn, imports of the oracle and torch) before timing."""
        self.pool.map(_warm, range(2 * self.workers), chunksize=1)

    def close(self):
        self.pool.close()
        self.pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
