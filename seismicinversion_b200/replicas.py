"""Replicas over several GPUs for the batched and served workloads.

Models of a batch and requests of a stream are independent, so several GPUs run replicas
with no inter-GPU data on the compute path:

* ``partition_by_work`` splits a list of models into per-rank shards of balanced work
  (longest-processing-time first, on the cost the batch planner uses: interfaces x
  slownesses x frequencies, x4 for gradients);
* ``run_batch_shard`` runs one rank's shard as a ``ModelBatch`` on its own GPU (one process
  per GPU, ranks from ``torch.distributed``) and ``gather_small_results`` collects the small
  outputs (chi, gradients) on rank 0 -- R grids stay on the GPU that computed them;
* ``ReplicaRouter`` fronts one ``KennettServer`` per GPU and sends each request to the
  replica with the least outstanding work; each result is that replica's, bit for bit the
  single-GPU result.

The reference has no multi-device path (its CPU gather uses a process pool,
``Kennett_Reflectivity/kennett_gather.py:246-288``).
"""

from __future__ import annotations

import heapq
import threading

import numpy as np

__all__ = ["model_cost", "partition_by_work", "run_batch_shard", "gather_small_results",
           "ReplicaRouter"]


def model_cost(n_layers: int, n_p: int, n_w: int, gradient: bool) -> float:
    """Work of one model as the batch planner weighs it: (omega, p, interface) updates, x4 for
    forward + gradient."""
    return float(max(n_layers - 1, 1)) * n_p * n_w * (4.0 if gradient else 1.0)


def partition_by_work(costs, n_shards: int) -> list[list[int]]:
    """Indices of ``costs`` split into ``n_shards`` shards of balanced total cost: the largest
    first, each to the currently lightest shard (ties: lowest shard).  Every index appears in
    exactly one shard, in ascending order within it; deterministic."""
    if n_shards < 1:
        raise ValueError("n_shards must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, s) for s in range(n_shards)]
    shards: list[list[int]] = [[] for _ in range(n_shards)]
    for i in order:
        load, s = heapq.heappop(heap)
        shards[s].append(i)
        heapq.heappush(heap, (load + float(costs[i]), s))
    return [sorted(sh) for sh in shards]


def _item_cost(it) -> float:
    from .layer_model import pack_layers

    L = pack_layers(it.model).shape[1]
    return model_cost(L, len(np.atleast_1d(it.p)), len(np.atleast_1d(it.omega)), it.gradient)


def run_batch_shard(items, rank: int, world: int, device=None, schedule=None, compute=None):
    """Runs this rank's shard of ``items`` (``BatchItem`` list, the same on every rank).

    Returns ``(indices, results)``: the global indices of the shard and, per index, a dict
    with ``R`` (device tensor, forward models and ``store_R``) and ``chi`` / ``grad`` (gradient
    models).  ``compute(items) -> list of dicts`` replaces the GPU batch (host-side tests)."""
    shards = partition_by_work([_item_cost(it) for it in items], world)
    idx = shards[rank]
    mine = [items[i] for i in idx]
    if compute is not None:
        return idx, compute(mine)
    from .batch import ModelBatch

    if not mine:
        return idx, []
    batch = ModelBatch(mine, schedule=schedule, device=device)
    batch.launch()
    out = []
    for b, it in enumerate(mine):
        res = {}
        if (not it.gradient) or it.store_R:
            res["R"] = batch.reflectivity(b)
        if it.gradient:
            chi, g = batch.misfit_gradient(b)
            res["chi"], res["grad"] = chi, g
        out.append(res)
    return idx, out


def gather_small_results(indices, results, n_items: int, group=None):
    """All-gathers the per-model chi and gradient (host copies) of every rank's shard, so every
    rank can return them in the caller's order: list of ``n_items`` dicts (``chi``, ``grad``
    numpy, or empty for forward models).  Uses ``torch.distributed.all_gather_object``."""
    import torch.distributed as dist

    small = []
    for i, r in zip(indices, results):
        d = {}
        if "chi" in r:
            d["chi"] = float(r["chi"])
            g = r["grad"]
            d["grad"] = g.detach().cpu().numpy() if hasattr(g, "detach") else np.asarray(g)
        small.append((i, d))
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, small, group=group)
    out = [dict() for _ in range(n_items)]
    for part in parts:
        for i, d in part:
            out[i] = d
    return out


class ReplicaRouter:
    """Least-outstanding-work request routing over several ``KennettServer`` replicas (one per
    GPU).  ``submit`` has the server's signature and returns the replica's ``Request``; a
    request's outstanding work is released when it completes."""

    def __init__(self, servers):
        if not servers:
            raise ValueError("ReplicaRouter needs at least one server")
        self.servers = list(servers)
        self._load = [0.0] * len(self.servers)
        self._lock = threading.Lock()
        self.routed = [0] * len(self.servers)

    def submit(self, model, p, omega, gradient: bool = False, R_obs=None,
               free_surface: bool = False):
        cost = model_cost(model.n_layers, len(p), len(omega), gradient)
        with self._lock:
            k = min(range(len(self.servers)), key=lambda s: (self._load[s], s))
            self._load[k] += cost
            self.routed[k] += 1
        req = self.servers[k].submit(model, p, omega, gradient=gradient, R_obs=R_obs,
                                     free_surface=free_surface)
        req.replica = k

        def release(_req, _k=k, _c=cost):
            with self._lock:
                self._load[_k] -= _c

        req.add_done_callback(release)
        return req

    @property
    def outstanding(self) -> list[float]:
        """Work submitted to each replica and not yet done."""
        with self._lock:
            return list(self._load)

    def close(self) -> None:
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
