"""Replicas on the GPU (one device standing in for two): the two ranks' shards of a batch give
every model the single-batch result (forward bit-identical; gradients to 1e-12, the batch
adds block partials with FP64 atomics), and the router over two GPU servers gives every
request the single-call result (forward bit-identical; gradients to 1e-11: the batch and the
single call sum the same per-frequency terms in different orders, and these gradients are
sums with cancellation, so their rounding differs at ~1e-12 of max |g|)."""

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _items():
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.batch import BatchItem
    from seismicinversion_b200.earth_models import uneven_batch_specs

    items = []
    for b, (m, p, w) in enumerate(uneven_batch_specs(24, seed=17, nw_choices=(64, 256),
                                                     np_range=(4, 24))):
        if b % 2:
            R_obs = D.reflectivity(D.layer_table(m), p, w) * 1.02
            items.append(BatchItem(m, p, w, gradient=True, R_obs=R_obs, store_R=True))
        else:
            items.append(BatchItem(m, p, w))
    return items


def test_batch_shards_equal_one_batch():
    from seismicinversion_b200.batch import ModelBatch
    from seismicinversion_b200.replicas import run_batch_shard

    items = _items()
    whole = ModelBatch(items)
    whole.launch()
    got = {}
    for rank in range(2):
        idx, res = run_batch_shard(items, rank, 2)
        for i, r in zip(idx, res):
            got[i] = r
    torch.cuda.synchronize()
    assert sorted(got) == list(range(len(items)))
    for i, it in enumerate(items):
        assert torch.equal(got[i]["R"], whole.reflectivity(i))
        if it.gradient:
            chi, g = whole.misfit_gradient(i)
            assert rel_err(got[i]["grad"].cpu().numpy(), g.cpu().numpy()) < 1e-12
            assert abs(float(got[i]["chi"]) - float(chi)) <= 1e-12 * abs(float(chi))


def test_router_over_two_gpu_servers():
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.replicas import ReplicaRouter
    from seismicinversion_b200.serve import KennettServer

    items = _items()
    with ReplicaRouter([KennettServer(max_batch_requests=8), KennettServer(max_batch_requests=8)]) as rt:
        reqs = [rt.submit(it.model, it.p, it.omega, gradient=it.gradient, R_obs=it.R_obs)
                for it in items]
        res = [r.wait(60) for r in reqs]
    assert all(c > 0 for c in rt.routed)
    for it, r in zip(items, res):
        tab = D.layer_table(it.model)
        if it.gradient:
            out, R = D.misfit_gradient(tab, it.p, it.omega, it.R_obs, want_R=True)
            L = it.model.n_layers
            assert rel_err(r["grad"].cpu().numpy(), out[:4 * L].cpu().numpy()) < 1e-11
            assert torch.equal(r["R"], R)
        else:
            assert torch.equal(r["R"], D.reflectivity(tab, it.p, it.omega))
    for r in reqs:
        r.release()
