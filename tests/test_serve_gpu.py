"""Serving on the GPU: a Poisson-like mix of forward and forward+gradient requests of uneven
size; every result equals the single-call entry point (forward bit-identical, gradient
1e-12), and one request gives the same result alone and inside the mix."""

import time

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _requests(n, seed):
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import uneven_batch_specs

    specs = uneven_batch_specs(n, seed=seed, nw_choices=(64, 128, 256), np_range=(4, 32))
    out = []
    for b, (m, p, w) in enumerate(specs):
        grad = b % 2 == 1
        obs = D.reflectivity(D.layer_table(m), p, w).cpu().numpy() * 0.98 if grad else None
        out.append((m, p, w, grad, obs))
    return out


def _check(req):
    from seismicinversion_b200 import device as D

    res = req.wait(60)
    tab = D.layer_table(req.model)
    if req.gradient:
        out, R = D.misfit_gradient(tab, req.p, req.omega, req.R_obs, want_R=True)
        L = req.model.n_layers
        assert rel_err(res["grad"].cpu().numpy(), out[:4 * L].cpu().numpy()) < 1e-12
        assert torch.equal(res["R"], R)
    else:
        assert torch.equal(res["R"], D.reflectivity(tab, req.p, req.omega))
    return res


def test_mix_matches_single_calls_and_alone_vs_mix():
    from seismicinversion_b200.serve import KennettServer

    reqs = _requests(60, seed=5)
    with KennettServer(max_batch_requests=16, max_inflight=2) as srv:
        # the probe request, alone
        m, p, w, g, o = reqs[1]
        alone = srv.submit(m, p, w, gradient=g, R_obs=o)
        a = _check(alone)
        # ... and inside a stream of arrivals (exponential gaps, ~5k req/s)
        rng = np.random.default_rng(0)
        handles = []
        for k, (m2, p2, w2, g2, o2) in enumerate(reqs):
            handles.append(srv.submit(m2, p2, w2, gradient=g2, R_obs=o2))
            time.sleep(rng.exponential(2e-4))
        for h in handles:
            _check(h)
        mixed = handles[1]
        assert rel_err(mixed.result["grad"].cpu().numpy(), a["grad"].cpu().numpy()) < 1e-12
        assert torch.equal(mixed.result["R"], a["R"])
        st = srv.stats()
        assert st["completed"] == 61 and st["batches"] >= 2


def test_single_request_group_runs_the_single_model_kernels():
    """A group of one request runs the single-model entry points: results identical to the
    direct call, bit for bit (gradient included)."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.serve import GpuBatchExecutor, KennettServer

    (m, p, w, _, _), (m1, p1, w1, g1, o1) = _requests(2, seed=9)
    ex = GpuBatchExecutor(n_streams=2)
    with KennettServer(executor=ex, max_batch_requests=16) as srv:
        res = srv.submit(m1, p1, w1, gradient=g1, R_obs=o1).wait(60)
        fwd = srv.submit(m, p, w).wait(60)
    tab = D.layer_table(m1)
    out, R = D.misfit_gradient(tab, p1, w1, o1, want_R=True)
    L = m1.n_layers
    assert g1 and torch.equal(res["grad"], out[:4 * L]) and torch.equal(res["R"], R)
    assert float(res["chi"]) == float(out[4 * L])
    assert torch.equal(fwd["R"], D.reflectivity(D.layer_table(m), p, w))


def test_small_groups_run_the_single_model_kernels():
    """A group of up to four requests (the default threshold) runs each request through the
    single-model entry points, one after another on the group's stream: no batch plan, and
    every result equals the direct call bit for bit."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.serve import GpuBatchExecutor, Request

    reqs = [Request(m, np.asarray(p, dtype=np.float64), np.asarray(w, dtype=np.complex128), g, o)
            for (m, p, w, g, o) in _requests(4, seed=11)]
    ex = GpuBatchExecutor(n_streams=1)
    handle = ex.launch(reqs)
    handle[1].synchronize()
    assert handle[0] is None  # no ModelBatch was built
    res = ex.results(handle, reqs)
    for r, x in zip(reqs, res):
        tab = D.layer_table(r.model)
        if r.gradient:
            out, R = D.misfit_gradient(tab, r.p, r.omega, r.R_obs, want_R=True)
            L = r.model.n_layers
            assert torch.equal(x["grad"], out[:4 * L]) and torch.equal(x["R"], R)
        else:
            assert torch.equal(x["R"], D.reflectivity(tab, r.p, r.omega))
