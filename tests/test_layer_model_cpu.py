"""Model validation on the host, with the reference's exceptions (layer_model.py:105-123:
ValueError for non-physical models) and the kernels' own limits (acoustic ocean, finite
parameters, positive Q, half-space conventions)."""

import numpy as np
import pytest

from seismicinversion_b200.earth_models import default_ocean_crust_model
from seismicinversion_b200.layer_model import LayerModel, complex_slowness, pack_layers


def _args(**kw):
    m = default_ocean_crust_model()
    a = dict(alpha=m.alpha, beta=m.beta, rho=m.rho, thickness=m.thickness, Q_alpha=m.Q_alpha,
             Q_beta=m.Q_beta)
    a.update(kw)
    return a


@pytest.mark.parametrize("kw,match", [
    (dict(alpha=[1.5, -1.6, 3.0, 5.0, 2.2]), "alpha"),
    (dict(beta=[0.0, -0.3, 1.5, 3.0, 1.1]), "beta"),
    (dict(rho=[1.0, 2.0, 0.0, 3.0, 1.8]), "rho"),
    (dict(rho=[1.0, 2.0, 3.0]), "length"),
])
def test_reference_validation(kw, match):
    with pytest.raises(ValueError, match=match):
        LayerModel(**_args(**kw))


@pytest.mark.parametrize("kw,match", [
    (dict(beta=[0.2, 0.3, 1.5, 3.0, 1.1]), "acoustic"),
    (dict(Q_alpha=[2e4, 100, 0.0, 100, 100]), "Q_alpha"),
    (dict(Q_beta=[1e10, 100, -1.0, 100, 100]), "Q_beta"),
    (dict(alpha=[1.5, np.inf, 3.0, 5.0, 2.2]), "finite"),
    (dict(thickness=[2.0, -1.0, 1.0, 1.0, np.inf]), "thickness"),
])
def test_kernel_limits(kw, match):
    with pytest.raises(ValueError, match=match):
        pack_layers(LayerModel(**_args(**kw)))


def test_half_space_conventions_and_layout():
    m = default_ocean_crust_model()
    tab = pack_layers(m)
    assert tab.shape == (6, m.n_layers) and tab.dtype == np.float64
    assert np.array_equal(tab[0], m.alpha) and np.array_equal(tab[3][:-1], m.thickness[:-1])
    # +inf and the torch path's 1e30 sentinel are both accepted for the half-space
    pack_layers(LayerModel(**_args(thickness=[2.0, 1.0, 1.0, 1.0, 1e30])))
    with pytest.raises(ValueError):
        complex_slowness(0.0, 100.0)
    with pytest.raises(ValueError):
        complex_slowness(1.5, 0.0)


@pytest.mark.parametrize("n_sub,seed", [(5, 0), (20, 1), (20, 2), (63, 3)])
def test_random_model_generator(n_sub, seed):
    """The seeded benchmark models: 1 km water (Vp 1.5, Vs 0, rho 1.0) over n_sub layers with
    Vp ~ U(1.8, 5.0) increasing with depth, Vs = Vp / U(1.7, 2.0), rho = 0.31 (1000 Vp)^0.25,
    h ~ U(0.2, 1.0), an infinite half-space, Q_alpha = 100 and Q_beta = 50; the same seed gives
    the same model."""
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=seed)
    assert m.n_layers == n_sub + 1
    assert (m.alpha[0], m.beta[0], m.rho[0], m.thickness[0]) == (1.5, 0.0, 1.0, 1.0)
    vp, vs = m.alpha[1:], m.beta[1:]
    assert np.all(np.diff(vp) >= 0) and np.all((vp >= 1.8) & (vp <= 5.0))
    assert np.all((vp / vs >= 1.7) & (vp / vs <= 2.0))
    assert np.allclose(m.rho[1:], 0.31 * (1000.0 * vp) ** 0.25, rtol=0, atol=1e-15)
    assert np.all((m.thickness[1:-1] >= 0.2) & (m.thickness[1:-1] <= 1.0))
    assert np.isinf(m.thickness[-1])
    assert np.all(m.Q_alpha == 100.0) and np.all(m.Q_beta == 50.0)
    m2 = random_layered_model(n_sub, seed=seed)
    assert all(np.array_equal(getattr(m, k), getattr(m2, k))
               for k in ("alpha", "beta", "rho", "thickness"))


def test_uneven_batch_workload():
    """The uneven-batching workload: total layers U{3..64}, n_omega in {256, 512, 1024, 2048}
    with omega_k = k 2 pi / 64, n_p U{16..256} with p_j = j 0.8 / n_p; seeded."""
    from seismicinversion_b200.earth_models import uneven_batch_specs

    specs = uneven_batch_specs(512, seed=3)
    Ls = np.array([m.n_layers for m, _, _ in specs])
    assert Ls.min() >= 3 and Ls.max() <= 64 and len(set(Ls)) > 40
    for m, p, w in specs[:64]:
        assert len(w) in (256, 512, 1024, 2048)
        assert np.allclose(w, np.arange(1, len(w) + 1) * (2 * np.pi / 64), rtol=0, atol=0)
        assert 16 <= len(p) <= 256 and p[-1] == pytest.approx(0.8)
        assert np.allclose(np.diff(p), 0.8 / len(p))
    again = uneven_batch_specs(512, seed=3)
    assert all(np.array_equal(a[0].alpha, b[0].alpha) for a, b in zip(specs, again))
