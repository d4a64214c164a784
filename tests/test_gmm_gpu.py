"""Global Matrix Method forward on the GPU (kr_gmm_reflectivity and its drop-ins).

References: the reference's own GMM outputs (golden vectors from
``GlobalMatrix.global_matrix.gmm_reflectivity`` and ``gmm_torch.gmm_reflectivity_torch``),
the GMM oracle, and the Kennett kernel (the reference's tests hold GMM and Kennett equal to
1e-10, ``GlobalMatrix/test_gmm.py:27-42``).
"""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import gmm_oracle as G
from oracle import kennett_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _model(g, tag):
    from seismicinversion_b200.layer_model import LayerModel

    return LayerModel(*[g[f"{tag}_{k}"] for k in ("alpha", "beta", "rho", "thickness",
                                                   "Q_alpha", "Q_beta")])


@pytest.mark.parametrize("tag", ["default", "two", "three", "c1"])
def test_vs_reference_gmm(golden, tag):
    from seismicinversion_b200 import device as D

    g = golden("gmm_reflectivity.npz")
    m = _model(g, tag)
    for fs in (False, True):
        R = D.gmm_reflectivity(D.layer_table(m), g[f"{tag}_p"], g[f"{tag}_omega"], fs)
        assert rel_err(R.cpu().numpy(), g[f"{tag}_R_fs{int(fs)}"]) < TOL, (tag, fs)


def test_drop_in_signatures(golden):
    from seismicinversion_b200 import gmm_reflectivity, gmm_reflectivity_torch
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_torch import model_to_tensors

    g = golden("gmm_reflectivity.npz")
    m = _model(g, "default")
    R = gmm_reflectivity(m, 0.3, g["default_omega"], free_surface=True)
    assert R.dtype == np.complex128 and R.shape == (255,)
    assert rel_err(R, g["default_R_fs1"][1]) < TOL
    Rd = gmm_reflectivity(m, 0.1, g["default_omega"], solver="dense")
    assert rel_err(Rd, g["default_Rdense_fs0"][0]) < TOL
    with pytest.raises(ValueError):
        gmm_reflectivity(m, 0.1, g["default_omega"], solver="lu")
    # torch path: the reference's gmm_reflectivity_torch on the 21-layer inversion model
    t = model_to_tensors(random_layered_model(20, seed=2))
    w = torch.as_tensor(g["c2_torch_omega"])
    Rt = gmm_reflectivity_torch(**t, p=0.3, omega=w)
    assert rel_err(Rt.numpy(), g["c2_torch_R_p0.3"]) < TOL


def test_gradient_is_the_adjoint_of_the_same_function():
    """gmm_reflectivity_torch: GMM value, Kennett-adjoint derivative (autograd and jacrev)."""
    from seismicinversion_b200 import gmm_reflectivity_torch, kennett_reflectivity_torch
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_torch import model_to_tensors

    t = model_to_tensors(random_layered_model(6, seed=9))
    w = torch.arange(1, 40, dtype=torch.float64) * 0.25
    a = t["alpha"].clone().requires_grad_(True)
    Rg = gmm_reflectivity_torch(a, t["beta"], t["rho"], t["thickness"], t["Q_alpha"],
                                t["Q_beta"], 0.35, w)
    (Rg.abs() ** 2).sum().backward()
    b = t["alpha"].clone().requires_grad_(True)
    Rk = kennett_reflectivity_torch(b, t["beta"], t["rho"], t["thickness"], t["Q_alpha"],
                                    t["Q_beta"], 0.35, w)
    (Rk.abs() ** 2).sum().backward()
    assert rel_err(Rg.detach().numpy(), Rk.detach().numpy()) < TOL
    assert rel_err(a.grad.numpy(), b.grad.numpy()) < 1e-8


@pytest.mark.parametrize("n_sub", [1, 2, 5, 20, 40, 99])
def test_vs_oracle_and_kennett(n_sub):
    """Random models of 2 to 100 layers (those above 30 layers evaluate their phases
    directly), damped frequencies, both surface conditions."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=200 + n_sub)
    p = np.array([0.0, 0.05, 0.3, 0.62, 0.9])
    w = np.arange(1, 301) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    tab = D.layer_table(m)
    for fs in (False, True):
        R = D.gmm_reflectivity(tab, p, w, fs).cpu().numpy()
        Ro = G.gmm_reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p,
                                w, fs)
        Rk = D.reflectivity(tab, p, w, fs).cpu().numpy()
        for i in range(len(p)):
            assert rel_err(R[i], Ro[i]) < TOL, (n_sub, p[i], fs, rel_err(R[i], Ro[i]))
            assert rel_err(R[i], Rk[i]) < 1e-9, (n_sub, p[i], fs, rel_err(R[i], Rk[i]))


def test_full_gather_grid_agrees_with_kennett():
    """The 21-layer gather grid (8192 p x 2047 damped omega): the independent method agrees
    with the Kennett kernel on every slowness up to 1.0 s/km."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model

    m = random_layered_model(20, seed=1)
    _, omd, p, _, _, _ = damped_gather_grid(64.0, 2048, 8192, 1.2)
    tab = D.layer_table(m)
    pt = torch.as_tensor(p, device="cuda")
    wt = torch.as_tensor(omd, device="cuda")
    Rg = D.gmm_reflectivity(tab, pt, wt, True)
    Rk = D.reflectivity(tab, pt, wt, True)
    assert bool(torch.isfinite(torch.view_as_real(Rg)).all())
    sel = pt <= 1.0
    num = (Rg[sel] - Rk[sel]).abs().amax(dim=1)
    den = Rk[sel].abs().amax(dim=1)
    assert float((num / den).max()) < 1e-9


def test_table_and_direct_phases_agree():
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(12, seed=5)
    p = np.array([0.1, 0.45, 0.8])
    w = np.arange(1, 520) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    perm = np.arange(len(w))
    perm[0:-1:2], perm[1::2] = perm[1::2].copy(), perm[0:-1:2].copy()
    tab = D.layer_table(m)
    R_tab = D.gmm_reflectivity(tab, p, w, True).cpu().numpy()
    R_dir = D.gmm_reflectivity(tab, p, w[perm], True).cpu().numpy()[:, np.argsort(perm)]
    assert rel_err(R_tab, R_dir) < 1e-12


def test_edge_cases():
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(3, seed=1)
    tab = D.layer_table(m)
    assert D.gmm_reflectivity(tab, np.zeros(0), np.arange(1, 5.0)).shape == (0, 4)
    assert D.gmm_reflectivity(tab, np.array([0.2]), np.zeros(0)).shape == (1, 0)
    R = D.gmm_reflectivity(tab, np.array([0.2]), np.array([3.0])).cpu().numpy()
    Ro = G.gmm_reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, [0.2],
                            np.array([3.0]))
    assert rel_err(R, Ro) < TOL
