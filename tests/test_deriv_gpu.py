"""Parity of the derivative path: kr_jacobian / kr_misfit_gradient and the torch drop-ins.

References: the reference's torch.func.jacrev ``jacobian`` and ``hessian`` and its
``invert_taup`` run (golden vectors), plus central finite differences of the oracle.
Tolerances: Jacobian vs jacrev 1e-10 relative (both exact derivatives); gradient vs the
Jacobian contraction 1e-12; vs finite differences 1e-6; Hessian (tangent of the adjoint,
exact) vs torch.func.hessian 1e-10, vs central differences of the exact gradient at their
truncation error.
"""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import kennett_oracle as O

pytestmark = pytest.mark.gpu


def _m(g):
    from seismicinversion_b200.layer_model import LayerModel

    return LayerModel(*[g[k] for k in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta")])


def _tensors(m):
    from seismicinversion_b200.kennett_torch import model_to_tensors

    return model_to_tensors(m)


@pytest.mark.parametrize("p", [0.2, 0.4])
@pytest.mark.parametrize("fs", [False, True])
def test_jacobian_vs_reference_jacrev(golden, p, fs):
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.kennett_torch import jacobian

    g = golden("derivs_default.npz")
    t = _tensors(default_ocean_crust_model())
    J = jacobian(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"], p,
                 torch.as_tensor(g["omega"]), free_surface=fs)
    assert J.shape == (32, 15) and J.device.type == "cpu"
    assert rel_err(J.numpy(), g[f"J_p{p}_fs{int(fs)}"]) < 1e-10
    if not fs:
        assert rel_err(J.numpy(), g[f"F_p{p}"]) < 1e-10  # analytical Frechet as well


def test_jacobian_21_layers_and_torch_forward(golden):
    from seismicinversion_b200.kennett_torch import jacobian, kennett_reflectivity_torch

    g = golden("derivs_c2.npz")
    t = _tensors(_m(g))
    for p in (0.05, 0.3):
        R = kennett_reflectivity_torch(**t, p=p, omega=torch.as_tensor(g["omega"]))
        assert rel_err(R.numpy(), g[f"R_p{p}"]) < 1e-10
        J = jacobian(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"],
                     p, torch.as_tensor(g["omega"]))
        assert J.shape == (64, 79)
        assert rel_err(J.numpy(), g[f"J_p{p}"]) < 1e-10
    w1024 = torch.arange(1, 1025, dtype=torch.float64) * (2 * np.pi / 64)
    R = kennett_reflectivity_torch(**t, p=0.3, omega=w1024)
    assert rel_err(R.numpy(), g["R1024_p0.3"]) < 1e-10


def test_autograd_and_func_jacrev_through_function(golden):
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.kennett_torch import (
        _pack_params,
        _unpack_params,
        kennett_reflectivity_torch,
        model_to_tensors,
    )

    g = golden("derivs_default.npz")
    t = model_to_tensors(default_ocean_crust_model(), requires_grad=True)
    w = torch.as_tensor(g["omega"])
    R = kennett_reflectivity_torch(**t, p=0.2, omega=w)
    loss = (R.real**2 + R.imag**2).sum()
    loss.backward()
    Jg = g["J_p0.2_fs0"]  # packed: alpha_1..4, beta_1..4, rho_1..4, h_1..3
    grad_ref = 2 * (R.detach().numpy().conj()[:, None] * Jg).real.sum(0)
    got = np.concatenate([t["alpha"].grad[1:], t["beta"].grad[1:], t["rho"].grad[1:],
                          t["thickness"].grad[1:-1]])
    assert rel_err(got, grad_ref) < 1e-10
    # torch.func.jacrev through the Function, as the reference's jacobian() does it
    t2 = model_to_tensors(default_ocean_crust_model())
    m0 = _pack_params(t2["alpha"], t2["beta"], t2["rho"], t2["thickness"])

    def f(m):
        a, b, r, h = _unpack_params(m, t2["alpha"], t2["beta"], t2["rho"], t2["thickness"])
        return kennett_reflectivity_torch(a, b, r, h, t2["Q_alpha"], t2["Q_beta"], 0.2, w)

    Jr = torch.func.jacrev(lambda m: f(m).real)(m0) + 1j * torch.func.jacrev(lambda m: f(m).imag)(m0)
    assert rel_err(Jr.numpy(), Jg) < 1e-10


def test_misfit_gradient_vs_jacobian_and_fd():
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(6, seed=21)
    L = m.n_layers
    tab = D.layer_table(m)
    p = np.array([0.05, 0.22, 0.41, 0.7])
    w = np.arange(1, 300) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    for fs in (False, True):
        R_true = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p, w, fs)
        R_obs = R_true * (1 + 0.03 * np.cos(np.arange(w.size)))[None, :]
        out, R = D.misfit_gradient(tab, p, w, R_obs, fs, want_R=True)
        out = out.cpu().numpy()
        Rg, J = D.jacobian(tab, p, w, fs)
        r = Rg.cpu().numpy() - R_obs
        g_ref = 2 * (r.conj()[:, None, :] * J.cpu().numpy()).real.sum(axis=(0, 2))
        assert rel_err(out[:4 * L], g_ref) < 1e-12
        assert abs(out[4 * L] - O.misfit(R_true, R_obs)) / O.misfit(R_true, R_obs) < 1e-10
        assert rel_err(R.cpu().numpy(), R_true) < 1e-10
        # central differences of the oracle misfit on a few parameters
        base = [m.alpha, m.beta, m.rho, m.thickness]
        for k, l in [(0, 1), (1, 3), (2, 5), (3, 2), (0, 0), (2, 0), (3, 0)]:
            arrs = [b.copy() for b in base]
            d = 1e-6 * arrs[k][l]
            arrs[k][l] += d
            cp = O.misfit(O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, fs), R_obs)
            arrs[k][l] -= 2 * d
            cm = O.misfit(O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, fs), R_obs)
            fd = (cp - cm) / (2 * d)
            assert abs(out[k * L + l] - fd) / (np.max(np.abs(out[:4 * L])) + 1e-300) < 1e-6, (k, l)


@pytest.mark.parametrize("n_sub", [100, 199])
def test_deep_models_recomputed_segments(n_sub):
    """Models deeper than one 64-step tape (101 and 200 layers): the reverse sweep recomputes
    checkpointed segments.  Jacobian columns against central differences of the oracle, and
    the misfit gradient against the Jacobian contracted with the residual."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=40 + n_sub)
    L = m.n_layers
    tab = D.layer_table(m)
    p = np.array([0.08, 0.4])
    w = np.arange(1, 48) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    Rg, J = D.jacobian(tab, p, w, True)
    J = J.cpu().numpy()
    Ro = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p, w, True)
    assert rel_err(Rg.cpu().numpy(), Ro) < 1e-10
    base = [m.alpha, m.beta, m.rho, m.thickness]
    for k, l in [(0, 1), (1, L // 3), (2, L // 2), (3, L - 2), (0, L - 1), (2, L - 1)]:
        arrs = [b.copy() for b in base]
        d = 1e-4 * arrs[k][l]  # deep columns are small: a larger step keeps rounding noise down
        arrs[k][l] += d
        Rp = O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, True)
        arrs[k][l] -= 2 * d
        Rm = O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, True)
        fd = (Rp - Rm) / (2 * d)
        # deep layers barely move R (their column is ~1e-6 of the largest): compare each column
        # against the Jacobian's overall scale where the finite difference is only noise
        scale = max(np.max(np.abs(fd)), 1e-4 * np.max(np.abs(J)))
        err = np.max(np.abs(J[:, k * L + l] - fd)) / scale
        assert err < 1e-6, (k, l, err)
    R_obs = Ro * (1 + 0.02 * np.sin(np.arange(w.size)))[None, :]
    out, _ = D.misfit_gradient(tab, p, w, R_obs, True)
    r = Rg.cpu().numpy() - R_obs
    g_ref = 2 * (r.conj()[:, None, :] * J).real.sum(axis=(0, 2))
    assert rel_err(out.cpu().numpy()[:4 * L], g_ref) < 1e-12


def test_gradient_inversion_size_64p_1024w():
    """21-layer inversion model, 64 slownesses x 1024 frequencies in one launch: gradient
    entries vs central differences of the oracle misfit (subset of 8 slownesses for the
    FD cost), and the full-size gradient vs the Jacobian contraction."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    true = random_layered_model(20, seed=2)
    rng = np.random.default_rng(2)
    start = random_layered_model(20, seed=2)
    for name in ("alpha", "beta", "rho"):
        getattr(start, name)[1:] *= np.exp(0.1 * rng.standard_normal(20))
    start.thickness[1:-1] *= np.exp(0.1 * rng.standard_normal(19))
    L = true.n_layers
    p = np.linspace(0.05, 0.6, 64)
    w = np.arange(1, 1025) * (2 * np.pi / 64)
    tab_true, tab = D.layer_table(true), D.layer_table(start)
    R_obs = D.reflectivity(tab_true, p, w)
    out, _ = D.misfit_gradient(tab, p, w, R_obs)
    Rg, J = D.jacobian(tab, p, w)
    r = Rg - R_obs
    g_ref = (2 * (r.conj()[:, None, :] * J).real.sum(dim=(0, 2))).cpu().numpy()
    out = out.cpu().numpy()
    assert rel_err(out[:4 * L], g_ref) < 1e-12
    sub = np.arange(0, 64, 8)
    out_s, _ = D.misfit_gradient(tab, p[sub], w, R_obs[sub])
    out_s = out_s.cpu().numpy()
    Ro = R_obs[sub].cpu().numpy()
    base = [start.alpha, start.beta, start.rho, start.thickness]
    for k, l in [(0, 3), (1, 10), (2, 17), (3, 8)]:
        arrs = [b.copy() for b in base]
        d = 1e-6 * arrs[k][l]
        arrs[k][l] += d
        cp = O.misfit(O.reflectivity(*arrs, start.Q_alpha, start.Q_beta, p[sub], w), Ro)
        arrs[k][l] -= 2 * d
        cm = O.misfit(O.reflectivity(*arrs, start.Q_alpha, start.Q_beta, p[sub], w), Ro)
        fd = (cp - cm) / (2 * d)
        assert abs(out_s[k * L + l] - fd) / np.max(np.abs(out_s[:4 * L])) < 1e-6, (k, l)


def test_hessian_vs_reference(golden):
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.kennett_torch import hessian, model_to_tensors

    g = golden("derivs_default.npz")
    t = model_to_tensors(default_ocean_crust_model())
    a = t["alpha"].clone()
    a[1] *= 1.02
    H = hessian(a, t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"], 0.2,
                torch.as_tensor(g["omega"]), R_obs=torch.as_tensor(g["R_obs_p0.2"]))
    assert rel_err(H.cpu().numpy(), g["H_p0.2_alpha1x1.02"]) < 1e-10


def test_torch_func_hessian_through_function_is_exact(golden):
    """torch.func.hessian of the misfit built on kennett_reflectivity_torch -- the way the
    reference's hessian() and invert_taup take it (forward over reverse) -- equals the
    reference's own torch.func.hessian golden to 1e-10: the Jacobian output carries the
    second derivative as its tangent.  Reverse over reverse (double backward) agrees."""
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.kennett_torch import (_pack_params, _unpack_params,
                                                     kennett_reflectivity_torch, model_to_tensors)

    g = golden("derivs_default.npz")
    t = model_to_tensors(default_ocean_crust_model())
    t["alpha"] = t["alpha"].clone()
    t["alpha"][1] *= 1.02
    w = torch.as_tensor(g["omega"])
    R_obs = torch.as_tensor(g["R_obs_p0.2"])
    m0 = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"])

    def chi(m):
        a, b, r, h = _unpack_params(m, t["alpha"], t["beta"], t["rho"], t["thickness"])
        R = kennett_reflectivity_torch(a, b, r, h, t["Q_alpha"], t["Q_beta"], 0.2, w)
        res = R - R_obs
        return (res.real**2 + res.imag**2).sum()

    H = torch.func.hessian(chi)(m0)
    assert rel_err(H.numpy(), g["H_p0.2_alpha1x1.02"]) < 1e-10
    H2 = torch.autograd.functional.hessian(chi, m0)
    assert rel_err(H2.numpy(), g["H_p0.2_alpha1x1.02"]) < 1e-10


def test_hessian_free_surface_vs_gradient_differences():
    """hessian() with the free surface (exact, tangent of the adjoint) equals second-order
    central differences of the exact gradient within their O(d^2) error; the raw H e_j
    columns are symmetric to rounding without symmetrisation."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_torch import (_pack_params, hessian,
                                                     misfit_gradient_packed, model_to_tensors,
                                                     packed_index)

    m = random_layered_model(5, seed=8)
    t = model_to_tensors(m)
    w = torch.arange(1, 97, dtype=torch.float64) * (2 * np.pi / 64.0) + 1j * (np.pi / 64)
    args = (t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"], 0.3, w)
    R_obs = 0.9 * torch.as_tensor(O.reflectivity(*[x.numpy() for x in args[:6]], [0.3],
                                                  w.numpy(), True)[0])
    H = hessian(*args, R_obs=R_obs, free_surface=True).cpu().numpy()
    L = m.n_layers
    idx = packed_index(L)
    V = torch.zeros((len(idx), 4 * L), dtype=torch.float64)
    V[torch.arange(len(idx)), torch.as_tensor(idx)] = 1.0
    HV = D.misfit_hvp(D.layer_table(m), [0.3], w, R_obs.reshape(1, -1), V, True)
    Hraw = HV[:, idx].cpu().numpy()
    assert rel_err(Hraw, Hraw.T) < 1e-12
    m0 = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"]).numpy()
    Hs = np.empty_like(H)
    for j in range(len(m0)):
        d = 1e-5 * max(abs(m0[j]), 1e-3)
        mp, mm = m0.copy(), m0.copy()
        mp[j] += d
        mm[j] -= d
        gp = misfit_gradient_packed(mp, *args[:6], 0.3, w, R_obs, True)[1].cpu().numpy()
        gm = misfit_gradient_packed(mm, *args[:6], 0.3, w, R_obs, True)[1].cpu().numpy()
        Hs[:, j] = (gp - gm) / (2 * d)
    assert rel_err(H, 0.5 * (Hs + Hs.T)) < 1e-5


def test_exact_hessian_vs_fourth_order_differences_21_layers():
    """The tangent-of-adjoint Hessian of the tau-p misfit (21 layers, 79 packed parameters,
    damped grid, evanescent slownesses) equals fourth-order central differences of the exact
    gradient (truncation ~1e-10) to 1e-8."""
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_torch import _pack_params, model_to_tensors
    from seismicinversion_b200.taup_inversion import _Problem

    true = random_layered_model(20, seed=2)
    start = random_layered_model(20, seed=2)
    start.alpha[1:] *= np.exp(0.05 * np.sin(np.arange(20)))
    p = np.array([0.05, 0.2, 0.45, 0.6])
    w = torch.arange(1, 257, dtype=torch.float64) * (2 * np.pi / 64.0)
    from seismicinversion_b200 import device as D

    R_obs = D.reflectivity(D.layer_table(true), p, w)
    t = model_to_tensors(true)
    prob = _Problem(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"],
                    p, w, R_obs)
    ts = model_to_tensors(start)
    phys = _pack_params(ts["alpha"], ts["beta"], ts["rho"], ts["thickness"]).numpy()
    H = prob.hessian_exact(phys)
    H4 = prob.hessian_fd(phys, step=1e-4, stencil=4)
    assert H.shape == (79, 79)
    assert rel_err(H, H4) < 1e-8


@pytest.mark.parametrize("n_sub,fs", [(5, False), (20, True), (70, False)])
def test_jacobian_dot_vs_jacobian_differences(n_sub, fs):
    """kr_jacobian_dot (d/dv of dR/dtheta) equals central differences of kr_jacobian along v
    to their truncation error, for a shallow, a 21-layer (free surface) and a 72-layer model
    (the last recomputes checkpointed tape segments)."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=40 + n_sub)
    tab = D.layer_table(m)
    L = tab.shape[1]
    tab[3, -1] = 1e30
    p = torch.tensor([0.08, 0.3, 0.55, 0.9], dtype=torch.float64, device=tab.device)
    w = (torch.arange(1, 65, dtype=torch.float64, device=tab.device) * (2 * np.pi / 64)
         + 1j * (np.pi / 64))
    gen = torch.Generator(device="cpu").manual_seed(n_sub)
    scale = torch.cat([tab[0], tab[1], tab[2], torch.cat([tab[3, :-1],
                                                          torch.zeros(1, device=tab.device)])])
    V = torch.randn(2, 4 * L, dtype=torch.float64, generator=gen).to(tab.device) * scale
    V[:, L] = 0.0  # the ocean's beta stays 0
    Jd = D.jacobian_dot(tab, p, w, V, fs)
    assert Jd.shape == (2, 4, 4 * L, 64)
    for d in range(2):
        eps = 1e-6

        def shifted(s):
            t = tab.clone()
            t[0] += s * V[d, :L]
            t[1] += s * V[d, L:2 * L]
            t[2] += s * V[d, 2 * L:3 * L]
            t[3, :-1] += s * V[d, 3 * L:4 * L - 1]
            return t

        Jp = D.jacobian(shifted(eps), p, w, fs, want_R=False)[1]
        Jm = D.jacobian(shifted(-eps), p, w, fs, want_R=False)[1]
        fd = (Jp - Jm) / (2 * eps)
        assert rel_err(Jd[d].cpu().numpy(), fd.cpu().numpy()) < 1e-6


def test_batched_exact_hessian_matches_sequential_differences():
    """The 2P-model batched Hessian equals central differences of single gradient launches."""
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_torch import _pack_params, model_to_tensors
    from seismicinversion_b200.taup_inversion import _Problem

    m = random_layered_model(6, seed=4)
    t = model_to_tensors(m)
    p = np.array([0.05, 0.15, 0.3])
    w = torch.arange(1, 49, dtype=torch.float64) * (2 * np.pi / 64.0)
    tab = torch.stack([t[k] for k in ("alpha", "beta", "rho", "thickness", "Q_alpha",
                                      "Q_beta")]).cuda()
    from seismicinversion_b200 import device as D

    R_obs = D.reflectivity(tab, torch.as_tensor(p).cuda(), w.cuda().to(torch.complex128))
    prob = _Problem(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"],
                    p, w, R_obs)
    base = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"]).numpy()
    phys = base * np.exp(0.03 * np.sin(np.arange(len(base))))
    for _ in range(2):  # second call reuses the batch with updated layers
        H = prob.hessian_fd(phys)
        phys = phys * 1.01
    phys = phys / 1.01
    P = len(phys)
    Hs = np.empty((P, P))
    for j in range(P):
        d = 1e-5 * max(abs(phys[j]), 1e-3)
        mp, mm = phys.copy(), phys.copy()
        mp[j] += d
        mm[j] -= d
        Hs[:, j] = (prob.chi_grad(mp)[1] - prob.chi_grad(mm)[1]) / (2 * d)
    Hs = 0.5 * (Hs + Hs.T)
    # same step, different kernels: the gradients agree to rounding, amplified by 1 / (2 d)
    assert np.max(np.abs(H - Hs)) <= 1e-6 * np.max(np.abs(Hs))


def test_invert_taup_matches_reference_run(golden):
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.taup_inversion import invert_taup

    g = golden("invert_small.npz")
    res = invert_taup(default_ocean_crust_model(), [0.1, 0.2, 0.3, 0.4], nfreq=32,
                      perturbation=0.05, max_iter=30)
    assert res.converged and res.param_error_history[-1] < 1e-3
    assert np.allclose(res.initial_model.alpha, g["init_alpha"], rtol=1e-14)
    n = min(5, len(res.misfit_history), len(g["misfit"]))
    # identical start; the first LM iterates agree closely (exact vs finite-difference Hessian)
    assert abs(res.misfit_history[0] - g["misfit"][0]) / g["misfit"][0] < 1e-10
    for k in range(1, n):
        assert abs(res.param_error_history[k] - g["param_err"][k]) <= 1e-3 * g["param_err"][0]
    assert np.allclose(res.recovered_model.alpha, g["rec_alpha"], rtol=1e-5)
    assert np.allclose(res.recovered_model.thickness[:-1], g["rec_thickness"][:-1], rtol=1e-5)


def test_invert_taup_gauss_newton_converges():
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.taup_inversion import invert_taup

    res = invert_taup(default_ocean_crust_model(), [0.1, 0.2, 0.3, 0.4], nfreq=32,
                      perturbation=0.02, max_iter=20, hessian="gauss-newton")
    assert res.converged and res.param_error_history[-1] < 1e-6


@pytest.mark.parametrize("hessian", ["gauss-newton", "exact"])
def test_invert_taup_batch_matches_sequential(hessian):
    """K concurrent inversions with the LM state on the device follow the sequential
    invert_taup trajectories (same starts, same rules; gradients agree to ~1e-12, so the
    histories agree closely) and converge alike."""
    from seismicinversion_b200.earth_models import default_ocean_crust_model, random_layered_model
    from seismicinversion_b200.taup_batch import invert_taup_batch
    from seismicinversion_b200.taup_inversion import invert_taup

    models = [default_ocean_crust_model(), random_layered_model(4, seed=12),
              random_layered_model(4, seed=13)]
    ps = [0.1, 0.2, 0.3, 0.4]
    seeds = [42, 7, 8]
    res = invert_taup_batch(models, ps, nfreq=32, perturbation=0.03, max_iter=25, seeds=seeds,
                            hessian=hessian)
    for k, m in enumerate(models):
        ref = invert_taup(m, ps, nfreq=32, perturbation=0.03, max_iter=25, seed=seeds[k],
                          hessian=hessian)
        r = res[k]
        assert np.allclose(r.initial_model.alpha, ref.initial_model.alpha, rtol=1e-15)
        n = min(4, r.n_iterations, ref.n_iterations)
        for i in range(n):
            assert abs(r.misfit_history[i] - ref.misfit_history[i]) <= \
                1e-6 * ref.misfit_history[0], (k, i)
        # same outcome: converged alike, final errors alike, the same recovered model
        assert r.converged == ref.converged
        assert abs(r.param_error_history[-1] - ref.param_error_history[-1]) <= \
            0.05 * ref.param_error_history[0] + 1e-6, (k, r.param_error_history[-1],
                                                        ref.param_error_history[-1])
        assert np.allclose(r.recovered_model.alpha, ref.recovered_model.alpha, rtol=1e-3)


@pytest.mark.parametrize("fs", [False, True])
def test_vjp_kernel_vs_jacobian_contraction(fs):
    """kr_vjp with an arbitrary complex cotangent equals Re sum conj(gR) J (kr_jacobian) to
    1e-12, on a 21-layer model over an evanescent-reaching slowness range."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(20, seed=11)
    tab = D.layer_table(m)
    p = torch.linspace(0.02, 0.9, 37, dtype=torch.float64, device=tab.device)
    w = (torch.arange(1, 301, dtype=torch.float64, device=tab.device) * (2 * np.pi / 64)
         + 1j * (np.pi / 64))
    gen = torch.Generator(device="cpu").manual_seed(5)
    gR = torch.randn(37, 300, dtype=torch.complex128, generator=gen).to(tab.device)
    g, R = D.vjp(tab, p, w, gR, fs, want_R=True)
    R2, J = D.jacobian(tab, p, w, fs)
    want = (gR.conj().unsqueeze(1) * J).real.sum((0, 2))
    assert rel_err(g.cpu().numpy(), want.cpu().numpy()) < 1e-12
    assert torch.equal(R, R2)  # the same forward sweep
    # linearity in the cotangent, and zero for a zero cotangent
    g2, _ = D.vjp(tab, p, w, 2.5 * gR + 1j * gR, fs)
    assert rel_err(g2.cpu().numpy(), (2.5 * g).cpu().numpy()
                   + D.vjp(tab, p, w, 1j * gR, fs)[0].cpu().numpy()) < 1e-12
    z, _ = D.vjp(tab, p, w, torch.zeros_like(gR), fs)
    assert torch.count_nonzero(z) == 0


def test_torch_backward_at_gather_size_forms_no_jacobian():
    """kennett_reflectivity_torch with the 21-layer gather grid's 8192 slownesses x 2047
    damped frequencies backpropagates through the adjoint kernel: the Jacobian would be
    8192 x 84 x 2047 complex (22.5 GB); the backward's peak device memory stays below 1 GB
    above the inputs, and the gradient equals the Jacobian contraction accumulated over
    slowness chunks to 1e-12."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model
    from seismicinversion_b200.kennett_torch import kennett_reflectivity_torch, model_to_tensors

    dev = torch.device("cuda", 0)
    m = random_layered_model(20, seed=1)
    _, omd, p, _, _, _ = damped_gather_grid(64.0, 2048, 8192, 1.2)
    t = {k: v.to(dev) for k, v in model_to_tensors(m).items()}
    for k in ("alpha", "beta", "rho", "thickness"):
        t[k].requires_grad_(True)
    p_t = torch.as_tensor(p, device=dev)
    w_t = torch.as_tensor(omd, device=dev)
    gen = torch.Generator(device="cpu").manual_seed(9)
    gR = torch.randn(len(p), len(omd), dtype=torch.complex128, generator=gen).to(dev)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats(dev)
    base = torch.cuda.memory_allocated(dev)
    R = kennett_reflectivity_torch(**t, p=p_t, omega=w_t, free_surface=True)
    grads = torch.autograd.grad(R, [t["alpha"], t["beta"], t["rho"], t["thickness"]], gR)
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated(dev) - base
    assert peak < (1 << 30), f"backward used {peak / 2**30:.2f} GiB"
    got = torch.cat(grads).cpu().numpy()
    tab = D.layer_table(m, dev)
    want = torch.zeros(4 * tab.shape[1], dtype=torch.float64, device=dev)
    for j0 in range(0, len(p), 512):
        _, J = D.jacobian(tab, p_t[j0:j0 + 512], w_t, True, want_R=False)
        want += (gR[j0:j0 + 512].conj().unsqueeze(1) * J).real.sum((0, 2))
        del J
    assert rel_err(got, want.cpu().numpy()) < 1e-12


def test_c2_1024_jacobians_and_gradient_vs_reference(golden):
    """The tau-p inversion workload at its own size (21 layers, 79 packed parameters,
    1024 frequencies) from its lognormal start: kr_jacobian at 4 of the 64 slownesses against
    the reference's jacrev (1e-10), the misfit gradient over those slownesses against the
    reference's autograd gradient (1e-10), and the exact Hessian (tangent of the adjoint)
    against torch.func.hessian of the differentiable CPU oracle at one slowness (1e-10)."""
    from oracle import torch_oracle as T
    from seismicinversion_b200.kennett_torch import (_pack_params, _unpack_params, jacobian,
                                                     misfit_gradient_packed, model_to_tensors)
    from seismicinversion_b200.layer_model import LayerModel
    from seismicinversion_b200.taup_inversion import _Problem

    g = golden("derivs_c2_1024.npz")
    start = LayerModel(*[g["start_" + k] for k in ("alpha", "beta", "rho", "thickness",
                                                   "Q_alpha", "Q_beta")])
    t = model_to_tensors(start)
    om = torch.as_tensor(g["omega"])
    for k, p in enumerate(g["p"]):
        J = jacobian(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"],
                     t["Q_beta"], float(p), om)
        assert rel_err(J.numpy(), g[f"J_{k}"]) < 1e-10, k
    m0 = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"]).numpy()
    R_obs = np.stack([g[f"R_obs_{k}"] for k in range(4)])
    chi, grad = misfit_gradient_packed(m0, t["alpha"], t["beta"], t["rho"], t["thickness"],
                                       t["Q_alpha"], t["Q_beta"], g["p"], om, R_obs)
    assert abs(chi - float(g["chi"])) / float(g["chi"]) < 1e-10
    assert rel_err(grad.cpu().numpy(), g["grad"]) < 1e-10
    prob = _Problem(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"],
                    g["p"][2:3], om, R_obs[2:3])
    H = prob.hessian_exact(m0)
    m = torch.as_tensor(m0)

    def chi_cpu(mm):
        a, b, r, h = _unpack_params(mm, t["alpha"], t["beta"], t["rho"], t["thickness"])
        return T.misfit(T.reflectivity(a, b, r, h, t["Q_alpha"], t["Q_beta"], g["p"][2:3], om),
                        torch.as_tensor(R_obs[2:3]))

    H_ref = torch.func.hessian(chi_cpu)(m).numpy()
    assert rel_err(H, H_ref) < 1e-10


def test_invert_taup_trajectory_vs_reference_21_layers(golden):
    """invert_taup with the exact (tangent-of-adjoint) Hessian follows the reference's own
    invert_taup (torch.func.hessian per slowness) on the 21-layer inversion model from the
    same uniform +-10 % start, 16 slownesses x 64 frequencies, 10 iterations: the same start,
    misfits and parameter errors at every iteration to 1e-6 relative."""
    import os

    from conftest import GOLDEN
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.taup_inversion import invert_taup

    if not os.path.exists(GOLDEN / "invert_c2.npz"):
        pytest.skip("reference trajectory fixture not generated")
    g = golden("invert_c2.npz")
    res = invert_taup(random_layered_model(20, seed=2), list(np.linspace(0.05, 0.6, 16)),
                      nfreq=64, perturbation=0.1, max_iter=10, seed=42, tol=0.0)
    assert np.allclose(res.initial_model.alpha, g["init_alpha"], rtol=1e-14)
    n = int(g["n_iter"])
    assert res.n_iterations == n
    assert np.allclose(res.misfit_history, g["misfit"], rtol=1e-6, atol=0)
    assert np.allclose(res.param_error_history, g["param_err"], rtol=1e-6, atol=0)
    assert np.allclose(res.recovered_model.alpha, g["rec_alpha"], rtol=1e-6)


@pytest.mark.parametrize("n_sub,fs", [(60, False), (120, True)])
def test_deep_model_hvp_vs_gradient_differences(n_sub, fs):
    """kr_misfit_hvp on models deeper than one 32-step dual tape: 62 layers (the frequency-sum
    kernel, two recomputed segments) and 122 layers with the free surface (per-step fallback:
    its sums exceed shared memory; four segments).  H v against central differences of the
    exact gradient along v, to their truncation error."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(n_sub, seed=70 + n_sub)
    tab = D.layer_table(m)
    L = tab.shape[1]
    p = torch.tensor([0.1, 0.35], dtype=torch.float64, device=tab.device)
    w = (torch.arange(1, 49, dtype=torch.float64, device=tab.device) * (2 * np.pi / 64)
         + 1j * (np.pi / 64))
    R_obs = 0.95 * D.reflectivity(tab, p, w, fs)
    gen = torch.Generator(device="cpu").manual_seed(n_sub)
    scale = torch.cat([tab[0], tab[1], tab[2], torch.cat([tab[3, :-1],
                                                          torch.zeros(1, device=tab.device)])])
    V = torch.randn(2, 4 * L, dtype=torch.float64, generator=gen).to(tab.device) * scale
    V[:, L] = 0.0  # the ocean's beta stays 0
    HV = D.misfit_hvp(tab, p, w, R_obs, V, fs)
    for d in range(2):
        eps = 1e-6

        def grad(s):
            t = tab.clone()
            t[0] += s * V[d, :L]
            t[1] += s * V[d, L:2 * L]
            t[2] += s * V[d, 2 * L:3 * L]
            t[3, :-1] += s * V[d, 3 * L:4 * L - 1]
            return D.misfit_gradient(t, p, w, R_obs, fs)[0][:4 * L]

        fd = (grad(eps) - grad(-eps)) / (2 * eps)
        assert rel_err(HV[d].cpu().numpy(), fd.cpu().numpy()) < 1e-6, d


def test_derivative_entry_points_with_empty_grids():
    """Empty slowness or frequency grids and zero directions: gradients, VJPs and H v are
    zeros, Jacobians and their directional derivatives are empty, nothing raises."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(4, seed=3)
    tab = D.layer_table(m)
    L = tab.shape[1]
    V = torch.ones((3, 4 * L), dtype=torch.float64, device=tab.device)
    w = np.arange(1, 9) * 0.3 + 0.05j
    for p, om in ((np.zeros(0), w), (np.array([0.2, 0.3]), np.zeros(0, complex))):
        n_p, n_w = len(p), len(om)
        zeros = np.zeros((n_p, n_w), complex)
        out, R = D.misfit_gradient(tab, p, om, zeros, want_R=True)
        assert torch.count_nonzero(out) == 0 and out.shape == (4 * L + 1,)
        assert tuple(R.shape) == (n_p, n_w)
        g, _ = D.vjp(tab, p, om, zeros)
        assert torch.count_nonzero(g) == 0 and g.shape == (4 * L,)
        _, J = D.jacobian(tab, p, om, want_R=False)
        assert tuple(J.shape) == (n_p, 4 * L, n_w)
        HV = D.misfit_hvp(tab, p, om, zeros, V)
        assert torch.count_nonzero(HV) == 0 and tuple(HV.shape) == (3, 4 * L)
        assert tuple(D.jacobian_dot(tab, p, om, V).shape) == (3, n_p, 4 * L, n_w)
    p = np.array([0.2])
    R_obs = D.reflectivity(tab, p, w)
    assert tuple(D.misfit_hvp(tab, p, w, R_obs, V[:0]).shape) == (0, 4 * L)
    assert tuple(D.jacobian_dot(tab, p, w, V[:0]).shape) == (0, 1, 4 * L, len(w))
