"""Batched uneven models (kr_batch_*): every model's result equals the single-model entry
points (forward: bit-identical, same arithmetic; gradient: 1e-12 relative, the batch adds
block partials with atomics), for every schedule, through CUDA-graph replay and after
in-place parameter updates; a sample of the uneven-batching workload against the oracle."""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import kennett_oracle as O

pytestmark = pytest.mark.gpu


def _items(seed=0, n=36):
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.batch import BatchItem
    from seismicinversion_b200.earth_models import random_layered_model

    rng = np.random.default_rng(seed)
    items = []
    for b in range(n):
        n_sub = int(rng.choice([1, 2, 4, 20, 63]))
        m = random_layered_model(n_sub, seed=1000 + b)
        n_p = int(rng.choice([1, 3, 16]))
        n_w = int(rng.choice([1, 7, 256, 300]))
        p = np.sort(rng.uniform(0.0, 0.9, n_p))
        w = np.arange(1, n_w + 1) * (2 * np.pi / 64) + (1j * np.pi / 64 if b % 3 == 0 else 0)
        grad = b % 2 == 1
        fs = b % 4 == 0
        R_obs = None
        if grad:
            R_obs = D.reflectivity(D.layer_table(m), p, w, fs).cpu().numpy() * (1 + 0.05j)
        items.append(BatchItem(m, p, w, gradient=grad, R_obs=R_obs, free_surface=fs,
                               store_R=grad and b % 3 == 1))
    return items


def _check(batch, items):
    from seismicinversion_b200 import device as D

    for b, it in enumerate(items):
        tab = D.layer_table(it.model)
        R1 = D.reflectivity(tab, it.p, it.omega, it.free_surface)
        if not it.gradient:
            # same phase tiles and decisions as the per-model forward kernel: identical bits
            assert torch.equal(batch.reflectivity(b), R1), b
        if it.gradient:
            out, Rg = D.misfit_gradient(tab, it.p, it.omega, it.R_obs, it.free_surface,
                                        want_R=True)
            if it.store_R:
                # the adjoint sweep's own R: identical to the per-model adjoint call
                assert torch.equal(batch.reflectivity(b), Rg), b
                assert rel_err(batch.reflectivity(b).cpu().numpy(), R1.cpu().numpy()) < 1e-12
            chi, g = batch.misfit_gradient(b)
            L = it.model.n_layers
            assert abs(float(chi) - float(out[4 * L])) <= 1e-12 * abs(float(out[4 * L])), b
            assert rel_err(g.cpu().numpy(), out[:4 * L].cpu().numpy()) < 1e-12, b


@pytest.mark.parametrize("schedule", [(32, 64), (32, 100), (64, 64), (128, 256), (128, 512)])
def test_batch_matches_single_calls(schedule):
    from seismicinversion_b200.batch import ModelBatch

    items = _items()
    batch = ModelBatch(items, schedule=schedule)
    batch.launch()
    torch.cuda.synchronize()
    _check(batch, items)


def test_graph_replay_and_inplace_update():
    from seismicinversion_b200.batch import ModelBatch
    from seismicinversion_b200.layer_model import LayerModel

    items = _items(seed=1, n=20)
    batch = ModelBatch(items, schedule=(128, 128))
    batch.capture()
    batch.run()
    torch.cuda.synchronize()
    _check(batch, items)
    # perturb every model (same shapes), replay the same graph
    new = []
    for it in items:
        m = it.model
        new_m = LayerModel(m.alpha * 1.01, m.beta * 0.99, m.rho * 1.02, m.thickness, m.Q_alpha,
                           m.Q_beta)
        it.model = new_m
        new.append(new_m)
    batch.update_layers(new)
    batch.run()
    batch.run()
    torch.cuda.synchronize()
    _check(batch, items)


def test_uneven_workload_sample_vs_oracle():
    from seismicinversion_b200.batch import BatchItem, ModelBatch, autotune
    from seismicinversion_b200.earth_models import uneven_batch_specs

    specs = uneven_batch_specs(48, seed=3)
    items = [BatchItem(m, p, w) for (m, p, w) in specs]
    batch = ModelBatch(items)
    best, times = autotune(batch, reps=1)
    assert best in times and all(t > 0 for t in times.values())
    batch.launch()
    torch.cuda.synchronize()
    small = sorted(range(len(specs)), key=lambda b: specs[b][0].n_layers * len(specs[b][1]) * len(specs[b][2]))[:6]
    for b in small:
        m, p, w = specs[b]
        Ro = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p, w)
        Rb = batch.reflectivity(b).cpu().numpy()
        for j in range(len(p)):
            assert rel_err(Rb[j], Ro[j]) < 1e-10, (b, j)


def test_invalid_batches_rejected():
    from seismicinversion_b200.batch import BatchItem, ModelBatch
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(3, seed=0)
    with pytest.raises(ValueError):
        ModelBatch([BatchItem(m, np.array([0.1]), np.array([1.0]), gradient=True)])
    with pytest.raises(ValueError):
        ModelBatch([BatchItem(m, np.array([0.1]), np.array([1.0]))], schedule=(96, 128))


def test_largest_uneven_models_forward_and_gradient_vs_oracle():
    """The two largest models of the 4096-model uneven workload (seed 3; 64 and 61 layers,
    ~256 slownesses x 2048 frequencies), batched among small models, against the oracle at
    full size (a spawned process pool over the slownesses): the forward R grid to 1e-10; the
    gradient model's stored R to 1e-10, its chi to 1e-10 and four gradient components (a
    deep layer's alpha, beta, rho and h) to central differences of the oracle misfit, 1e-6."""
    from oracle.cpu_baseline import ReflectivityPool
    from seismicinversion_b200.batch import BatchItem, ModelBatch
    from seismicinversion_b200.earth_models import uneven_batch_specs
    from seismicinversion_b200.layer_model import LayerModel

    specs = uneven_batch_specs(4096, seed=3)
    order = sorted(range(len(specs)), key=lambda b: -(specs[b][0].n_layers * len(specs[b][1])
                                                      * len(specs[b][2])))
    fa, ga = order[0], order[1]
    mf, pf, wf = specs[fa]
    mg, pg, wg = specs[ga]
    assert mf.n_layers >= 61 and mg.n_layers >= 61 and len(wf) == len(wg) == 2048
    f = np.exp(0.03 * np.sin(np.arange(mg.n_layers)))
    perturbed = LayerModel(mg.alpha * f, mg.beta * f, mg.rho, mg.thickness, mg.Q_alpha, mg.Q_beta)
    with ReflectivityPool() as pool:
        Rf_o = pool.reflectivity(mf, pf, wf)
        R_obs = pool.reflectivity(perturbed, pg, wg)
        Rg_o = pool.reflectivity(mg, pg, wg)
        chi_o = float(np.sum(np.abs(Rg_o - R_obs) ** 2))
        L = mg.n_layers
        base = [mg.alpha, mg.beta, mg.rho, mg.thickness]
        fd = {}
        for k, l in [(0, L - 10), (1, L // 2), (2, 5), (3, L - 3)]:
            arrs = [b.copy() for b in base]
            d = 1e-6 * arrs[k][l]
            arrs[k][l] += d
            cp = np.sum(np.abs(pool.reflectivity(LayerModel(*arrs, mg.Q_alpha, mg.Q_beta), pg, wg)
                               - R_obs) ** 2)
            arrs[k][l] -= 2 * d
            cm = np.sum(np.abs(pool.reflectivity(LayerModel(*arrs, mg.Q_alpha, mg.Q_beta), pg, wg)
                               - R_obs) ** 2)
            fd[(k, l)] = (cp - cm) / (2 * d)
    small = [BatchItem(m, p, w) for (m, p, w) in specs[:8]]
    items = small + [BatchItem(mf, pf, wf),
                     BatchItem(mg, pg, wg, gradient=True, R_obs=R_obs, store_R=True)]
    batch = ModelBatch(items, schedule=(128, 2048))
    batch.launch()
    torch.cuda.synchronize()
    assert rel_err(batch.reflectivity(8).cpu().numpy(), Rf_o) < 1e-10
    assert rel_err(batch.reflectivity(9).cpu().numpy(), Rg_o) < 1e-10
    chi, g = batch.misfit_gradient(9)
    assert abs(float(chi) - chi_o) / chi_o < 1e-10
    g = g.cpu().numpy()
    for (k, l), v in fd.items():
        assert abs(g[k * L + l] - v) / np.max(np.abs(g)) < 1e-6, (k, l, g[k * L + l], v)
