"""Replicas for the batched and served workloads, host logic on the CPU: the work-balanced
partition of a batch over ranks, two gloo ranks each running their shard and all-gathering
the small results (identical to the single-process results), and the least-outstanding-work
router over two servers (each request's result is the single-server result).  The model
arithmetic is the oracle (test-only stand-in for the GPU batch)."""

import os
import socket
import threading
import time

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from seismicinversion_b200.replicas import ReplicaRouter, model_cost, partition_by_work


def test_partition_by_work_covers_and_balances():
    rng = np.random.default_rng(0)
    for n, world in ((0, 2), (1, 4), (7, 3), (400, 2), (4096, 8)):
        costs = rng.pareto(1.5, n) + 0.1
        shards = partition_by_work(costs, world)
        assert len(shards) == world
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(n))
        assert all(sh == sorted(sh) for sh in shards)
        if n:
            loads = [float(np.sum(costs[sh])) for sh in shards]
            # greedy LPT: no shard exceeds the mean by more than one item
            assert max(loads) <= np.sum(costs) / world + np.max(costs) + 1e-9
    assert partition_by_work([3.0, 1.0, 2.0], 2) == partition_by_work([3.0, 1.0, 2.0], 2)
    assert model_cost(21, 64, 1024, True) == 4 * model_cost(21, 64, 1024, False)


def _specs(n=12):
    from seismicinversion_b200.earth_models import uneven_batch_specs

    return uneven_batch_specs(n, seed=13, nw_choices=(8, 16), np_range=(2, 5))


def _items():
    from oracle import kennett_oracle as O
    from seismicinversion_b200.batch import BatchItem

    items = []
    for b, (m, p, w) in enumerate(_specs()):
        if b % 2:
            R_obs = 1.02 * O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha,
                                          m.Q_beta, p, w)
            items.append(BatchItem(m, p, w, gradient=True, R_obs=R_obs))
        else:
            items.append(BatchItem(m, p, w))
    return items


def oracle_compute(items):
    """Per item: chi and its finite-difference gradient in alpha (gradient items) or R."""
    from oracle import kennett_oracle as O

    out = []
    for it in items:
        m = it.model
        R = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, it.p,
                           it.omega)
        if not it.gradient:
            out.append({"R": R})
            continue
        g = np.zeros(m.n_layers)
        for l in range(m.n_layers):
            a = m.alpha.copy()
            d = 1e-6 * a[l]
            a[l] += d
            cp = O.misfit(O.reflectivity(a, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta,
                                         it.p, it.omega), it.R_obs)
            a[l] -= 2 * d
            cm = O.misfit(O.reflectivity(a, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta,
                                         it.p, it.omega), it.R_obs)
            g[l] = (cp - cm) / (2 * d)
        out.append({"chi": O.misfit(R, it.R_obs), "grad": g})
    return out


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from seismicinversion_b200.replicas import gather_small_results, run_batch_shard

        items = _items()
        idx, res = run_batch_shard(items, rank, world, compute=oracle_compute)
        small = gather_small_results(idx, res, len(items))
        out[rank] = (idx, small)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_a_batch_like_one_process():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    ref = oracle_compute(_items())
    idx0, idx1 = out[0][0], out[1][0]
    assert sorted(idx0 + idx1) == list(range(len(ref))) and idx0 and idx1
    for r in range(2):
        small = out[r][1]
        for i, want in enumerate(ref):
            if "chi" in want:
                assert small[i]["chi"] == want["chi"]
                assert np.array_equal(small[i]["grad"], want["grad"])
            else:
                assert small[i] == {}


class _FakeExecutor:
    """Completes each group after `delay` s with the oracle reflectivity of every request."""

    def __init__(self, delay):
        self.delay = delay
        self.seen = 0

    def launch(self, reqs):
        self.seen += len(reqs)
        return time.perf_counter() + self.delay

    def ready(self, h):
        return time.perf_counter() >= h

    def results(self, h, reqs):
        from oracle import kennett_oracle as O

        return [{"R": O.reflectivity(r.model.alpha, r.model.beta, r.model.rho,
                                     r.model.thickness, r.model.Q_alpha, r.model.Q_beta, r.p,
                                     r.omega)} for r in reqs]


def test_router_balances_and_returns_single_server_results():
    from seismicinversion_b200.serve import KennettServer

    specs = _specs(24)
    exs = [_FakeExecutor(0.01), _FakeExecutor(0.01)]
    with ReplicaRouter([KennettServer(executor=e, max_batch_requests=4) for e in exs]) as rt:
        reqs = [rt.submit(m, p, w) for (m, p, w) in specs]
        res = [r.wait(30)["R"] for r in reqs]
        deadline = time.time() + 5
        while any(abs(x) > 0 for x in rt.outstanding) and time.time() < deadline:
            time.sleep(0.01)
        assert rt.outstanding == [0.0, 0.0]
    assert exs[0].seen > 0 and exs[1].seen > 0 and sum(rt.routed) == len(specs)
    with KennettServer(executor=_FakeExecutor(0.0), max_batch_requests=4) as one:
        for (m, p, w), r in zip(specs, res):
            assert np.array_equal(one.submit(m, p, w).wait(30)["R"], r)


def test_done_callbacks_run_once_also_when_added_late():
    from seismicinversion_b200.serve import KennettServer

    (m, p, w), = _specs(1)
    seen = []
    lock = threading.Lock()
    with KennettServer(executor=_FakeExecutor(0.02)) as srv:
        r = srv.submit(m, p, w)
        r.add_done_callback(lambda q: seen.append(("early", q.id)))
        r.wait(10)
        r.add_done_callback(lambda q: seen.append(("late", q.id)))
        bad = srv.submit(m, [], w)  # rejected at once
        bad.add_done_callback(lambda q: seen.append(("rejected", q.error is not None)))
    with lock:
        assert sorted(seen) == sorted([("early", r.id), ("late", r.id), ("rejected", True)])
