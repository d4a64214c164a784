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
