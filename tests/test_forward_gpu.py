"""Parity of the fused forward kernel (kr_reflectivity) with the reference.

Golden vectors come from the reference itself; the oracle (a NumPy restatement pinned to
those vectors) covers sizes and models with no stored fixture.  Tolerance: 1e-10 relative
(max|x - ref| / max|ref|) -- the accuracy bar of the path -- except on the reference's
default model, where each slowness gets 10x the disagreement between the reference's own
two implementations (it reaches 8.8e-11 at p = 1.2), floored at 1e-10.
"""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import kennett_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _m(g, prefix=""):
    from seismicinversion_b200.layer_model import LayerModel

    return LayerModel(*[g[prefix + k] for k in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta")])


def _oracle(m, p, omega, fs):
    return O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p, omega, fs)


def test_c0_single_slowness(golden):
    from seismicinversion_b200 import kennett_reflectivity

    g = golden("c0_trace.npz")
    R = kennett_reflectivity(_m(g), float(g["p"]), g["omega"], free_surface=True)
    assert R.dtype == np.complex128 and R.shape == (2047,)
    assert rel_err(R, g["R"]) < TOL


@pytest.mark.parametrize("tag", ["real_fs0", "real_fs1", "damped_fs0", "damped_fs1"])
def test_default_model(golden, tag):
    from seismicinversion_b200 import kennett_reflectivity_batch

    g = golden("default_model_R.npz")
    R = kennett_reflectivity_batch(_m(g), g["p"], g["omega_" + tag], free_surface=tag.endswith("1"))
    for i, p in enumerate(g["p"]):
        tol = max(TOL, 10.0 * rel_err(g["Rb_" + tag][i], g["R_" + tag][i]))
        assert rel_err(R[i], g["R_" + tag][i]) < tol, (p, rel_err(R[i], g["R_" + tag][i]))


def test_c1_subset(golden):
    from seismicinversion_b200 import kennett_reflectivity_batch

    g = golden("c1_subset_R.npz")
    R = kennett_reflectivity_batch(_m(g), g["p"], g["omega"], free_surface=True)
    for i in range(len(g["p"])):
        assert rel_err(R[i], g["R"][i]) < TOL, (g["p"][i], rel_err(R[i], g["R"][i]))


def test_c1_full_grid_sampled_rows():
    """Full 8192 x 2047 grid of the 21-layer gather model: sampled rows vs the oracle, and
    every row of the batch equals the single-slowness call (same kernel, bit-identical)."""
    from seismicinversion_b200 import kennett_reflectivity
    from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model
    from seismicinversion_b200.kennett_reflectivity_gpu import kennett_reflectivity_batch

    m = random_layered_model(20, seed=1)
    om, omd, p, dp, taper, gamma = damped_gather_grid(64.0, 2048, 8192, 1.2)
    w = torch.as_tensor(omd, device="cuda")
    R = kennett_reflectivity_batch(m, torch.as_tensor(p, device="cuda"), w, free_surface=True)
    assert R.shape == (8192, 2047) and bool(torch.isfinite(torch.view_as_real(R)).all())
    rows = np.random.default_rng(5).choice(8192, 8, replace=False)
    Ro = _oracle(m, p[rows], omd, True)
    Rg = R[torch.as_tensor(rows, device="cuda")].cpu().numpy()
    for k in range(len(rows)):
        assert rel_err(Rg[k], Ro[k]) < TOL, (p[rows[k]], rel_err(Rg[k], Ro[k]))
    one = kennett_reflectivity(m, float(p[rows[0]]), w, free_surface=True)
    assert torch.equal(one, R[rows[0]])


def test_phase_table_and_direct_exponentials_agree():
    """Uniform frequency grids take the tabulated phase factors, non-uniform ones the direct
    exponentials: a grid with neighbours swapped in every tile (direct) matches the uniform
    grid (table) after unswapping; a descending grid and a grid with one perturbed tile also
    match the oracle."""
    from seismicinversion_b200 import kennett_reflectivity_batch
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(20, seed=1)
    p = np.array([0.0, 0.02, 0.3, 0.55, 0.8, 1.2])
    om = np.arange(1, 700) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    R_tab = kennett_reflectivity_batch(m, p, om, free_surface=True)
    perm = np.arange(len(om))
    perm[0:-1:2], perm[1::2] = perm[1::2].copy(), perm[0:-1:2].copy()
    R_dir = kennett_reflectivity_batch(m, p, om[perm], free_surface=True)[:, np.argsort(perm)]
    Ro = _oracle(m, p, om, True)
    for i in range(len(p)):
        assert rel_err(R_tab[i], Ro[i]) < TOL and rel_err(R_dir[i], Ro[i]) < TOL, p[i]
        assert rel_err(R_tab[i], R_dir[i]) < 1e-12, p[i]
    R_rev = kennett_reflectivity_batch(m, p, om[::-1].copy(), free_surface=True)[:, ::-1]
    om2 = om.copy()
    om2[300] += 1e-9
    R_pert = kennett_reflectivity_batch(m, p, om2, free_surface=True)
    Ro2 = _oracle(m, p, om2, True)
    for i in range(len(p)):
        assert rel_err(R_rev[i], Ro[i]) < TOL, p[i]
        assert rel_err(R_pert[i], Ro2[i]) < TOL, p[i]


@pytest.mark.parametrize("n_sub", [1, 2, 3, 8, 63, 255])
def test_layer_counts(n_sub):
    from seismicinversion_b200 import kennett_reflectivity_batch
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=100 + n_sub)
    p = np.array([0.0, 0.05, 0.3, 0.7, 1.1])
    om = np.arange(1, 130) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    for fs in (False, True):
        R = kennett_reflectivity_batch(m, p, om, free_surface=fs)
        Ro = _oracle(m, p, om, fs)
        for i in range(len(p)):
            assert rel_err(R[i], Ro[i]) < TOL, (n_sub, p[i], fs, rel_err(R[i], Ro[i]))


def test_edge_sizes_and_conventions():
    from seismicinversion_b200 import kennett_reflectivity, kennett_reflectivity_batch
    from seismicinversion_b200.earth_models import default_ocean_crust_model, random_layered_model

    m = random_layered_model(5, seed=0)
    # one frequency, one slowness
    R = kennett_reflectivity(m, 0.2, np.array([3.0]))
    assert R.shape == (1,) and rel_err(R, _oracle(m, [0.2], np.array([3.0]), False)[0]) < TOL
    # empty slowness / frequency grids
    assert kennett_reflectivity_batch(m, np.zeros(0), np.arange(1, 5.0)).shape == (0, 4)
    assert kennett_reflectivity_batch(m, np.array([0.1]), np.zeros(0)).shape == (1, 0)
    # half-space as +inf and as the torch 1e30 sentinel give identical results
    m2 = random_layered_model(5, seed=0)
    m2.thickness[-1] = 1e30
    om = np.arange(1, 300) * 0.1
    assert np.array_equal(kennett_reflectivity(m, 0.3, om), kennett_reflectivity(m2, 0.3, om))
    # ragged: a frequency count that is not a multiple of the block
    om = np.arange(1, 258) * 0.05
    assert rel_err(kennett_reflectivity(default_ocean_crust_model(), 0.25, om),
                   _oracle(default_ocean_crust_model(), [0.25], om, False)[0]) < TOL


def test_invalid_models_raise():
    from seismicinversion_b200 import kennett_reflectivity
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.layer_model import LayerModel

    m = random_layered_model(3, seed=1)
    bad = LayerModel(m.alpha, np.r_[0.3, m.beta[1:]], m.rho, m.thickness, m.Q_alpha, m.Q_beta)
    with pytest.raises(ValueError, match="acoustic"):
        kennett_reflectivity(bad, 0.2, np.arange(1, 5.0))
    big = random_layered_model(256, seed=2)  # 257 layers > KR_MAX_LAYERS
    with pytest.raises(ValueError):
        kennett_reflectivity(big, 0.2, np.arange(1, 5.0))


def test_device_tensors_stay_on_device():
    from seismicinversion_b200 import kennett_reflectivity_batch
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(5, seed=0)
    w = torch.arange(1, 100, device="cuda", dtype=torch.float64).to(torch.complex128) * 0.1
    R = kennett_reflectivity_batch(m, torch.tensor([0.1, 0.2], device="cuda", dtype=torch.float64), w)
    assert R.is_cuda and R.dtype == torch.complex128
    assert rel_err(R.cpu().numpy(), _oracle(m, [0.1, 0.2], w.cpu().numpy(), False)) < TOL


@pytest.mark.parametrize("n_sub", [20, 40])
def test_register_budget_variants_are_bit_identical(n_sub):
    """kr_set_forward_variant only changes the kernel's register budget: every setting gives
    the same bits (21 layers on the phase-table path, 41 layers on direct phases)."""
    from seismicinversion_b200 import _lib
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=11)
    p = np.linspace(0.01, 1.1, 37)
    w = np.arange(1, 700) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    tab = D.layer_table(m)
    h = _lib.lib()
    outs = []
    try:
        for v in (4, 5, 6, 0):
            h.kr_set_forward_variant(v)
            outs.append(D.reflectivity(tab, p, w, True).cpu().numpy())
    finally:
        h.kr_set_forward_variant(0)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    assert rel_err(outs[0], _oracle(m, p, w, True)) < TOL
