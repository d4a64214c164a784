"""Autograd / torch.func plumbing of the kennett_reflectivity_torch Function, on the CPU.

The device computation is replaced by an analytic stand-in with known first and second
derivatives (test-only monkeypatches of ``_compute``, ``_vjp`` and ``_jacobian_dot``), so the
routing of gradients, jacrev / jacfwd, vjp / jvp and the exactness of torch.func.hessian
(forward over reverse) and torch.autograd.functional.hessian (reverse over reverse) are
checked without a GPU.  The GPU tests check the real kernels through the same Function.
"""

import numpy as np
import pytest
import torch

import seismicinversion_b200.kennett_torch as KT


def _plain(*args):
    """The kernels read raw device memory: like them, the stand-ins refuse tensors that a
    torch.func transform has wrapped."""
    for a in args:
        if isinstance(a, torch.Tensor):
            assert not torch._C._functorch.is_functorch_wrapped_tensor(a), "wrapped tensor"


def _fake_compute(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, need_jac):
    # R(w) = sum_k sum_l c[k, l](w) * x_k[l]^2  (nonlinear, known derivative)
    _plain(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega)
    xs = [torch.as_tensor(t, dtype=torch.float64).detach() for t in (alpha, beta, rho, thickness)]
    L = xs[0].shape[0]
    w = torch.as_tensor(omega).detach().to(torch.complex128)
    p_t = torch.as_tensor(p, dtype=torch.float64).reshape(-1)
    R = torch.zeros((p_t.numel(), w.numel()), dtype=torch.complex128)
    J = torch.zeros((p_t.numel(), 4 * L, w.numel()), dtype=torch.complex128)
    for j, pj in enumerate(p_t):
        for k, x in enumerate(xs):
            for l in range(L):
                c = torch.exp(1j * w * (0.1 * (l + 1) + 0.01 * k)) * (1 + pj)
                R[j] += c * x[l] ** 2
                J[j, k * L + l] = c * 2 * x[l]
    return R, (J if need_jac else None)


CALLS = []


def _recording_compute(*args):
    CALLS.append(("compute", bool(args[-1])))
    return _fake_compute(*args)


def _fake_vjp(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, gR):
    _plain(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, gR)
    CALLS.append(("vjp", tuple(gR.shape)))
    _, J = _fake_compute(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, True)
    g = gR.reshape(J.shape[0], -1).conj().unsqueeze(-2) * J
    return g.real.sum(-1).sum(0)


def _fake_jacobian_dot(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, V):
    # d/dv of J[k L + l] = 2 c[k, l] x_k[l]  is  2 c[k, l] v[k L + l]
    _plain(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, V)
    CALLS.append(("jdot", int(V.shape[0])))
    L = torch.as_tensor(alpha).shape[0]
    w = torch.as_tensor(omega).detach().to(torch.complex128)
    p_t = torch.as_tensor(p, dtype=torch.float64).reshape(-1)
    V = torch.as_tensor(V, dtype=torch.float64).reshape(-1, 4 * L)
    out = torch.zeros((V.shape[0], p_t.numel(), 4 * L, w.numel()), dtype=torch.complex128)
    for j, pj in enumerate(p_t):
        for k in range(4):
            for l in range(L):
                c = torch.exp(1j * w * (0.1 * (l + 1) + 0.01 * k)) * (1 + pj)
                out[:, j, k * L + l] = 2 * c * V[:, k * L + l, None]
    return out


@pytest.fixture
def fake(monkeypatch):
    CALLS.clear()
    monkeypatch.setattr(KT, "_compute", _recording_compute)
    monkeypatch.setattr(KT, "_vjp", _fake_vjp)
    monkeypatch.setattr(KT, "_jacobian_dot", _fake_jacobian_dot)


def _model():
    t = KT.model_to_tensors(
        __import__("seismicinversion_b200.earth_models", fromlist=["x"]).random_layered_model(3, 1))
    return t


def test_backward_matches_jacobian(fake):
    t = _model()
    for k in ("alpha", "beta", "rho", "thickness"):
        t[k] = t[k].clone().requires_grad_(True)
    t["thickness"] = t["thickness"].detach().clone()
    t["thickness"][-1] = 5.0
    t["thickness"].requires_grad_(True)
    w = torch.arange(1, 9, dtype=torch.float64) * 0.5
    R = KT.kennett_reflectivity_torch(**t, p=0.2, omega=w)
    loss = (R.real**2 + R.imag**2).sum()
    loss.backward()
    Rf, J = _fake_compute(t["alpha"], t["beta"], t["rho"], t["thickness"], 0, 0, 0.2, w, False, True)
    L = t["alpha"].shape[0]
    g = (2 * Rf[0].conj().unsqueeze(0) * J[0]).real.sum(-1)
    for k, name in enumerate(("alpha", "beta", "rho", "thickness")):
        assert torch.allclose(t[name].grad, g[k * L:(k + 1) * L], rtol=1e-12, atol=1e-12)
    # plain autograd: the forward formed no Jacobian and backward ran the VJP entry point
    assert CALLS[0] == ("compute", False)
    assert ("vjp", (8,)) in CALLS and ("compute", True) not in CALLS


def test_inference_forms_no_jacobian(fake):
    t = _model()
    w = torch.arange(1, 9, dtype=torch.float64) * 0.5
    p = torch.tensor([0.1, 0.2, 0.3], dtype=torch.float64)
    R = KT.kennett_reflectivity_torch(**t, p=p, omega=w)
    assert R.shape == (3, 8)
    assert CALLS == [("compute", False)]
    _, J = KT._KennettFunction.apply(*(t[k] for k in ("alpha", "beta", "rho", "thickness",
                                                      "Q_alpha", "Q_beta")), p, w, False, KT._NONE)
    assert J.numel() == 0  # no Jacobian placeholder of size n_p x 4L x n_w


def test_vector_p_backward_and_double_backward(fake):
    t = _model()
    for k in ("alpha", "beta", "rho"):
        t[k] = t[k].clone().requires_grad_(True)
    w = torch.arange(1, 7, dtype=torch.float64) * 0.4
    p = torch.tensor([0.1, 0.25], dtype=torch.float64)
    R = KT.kennett_reflectivity_torch(**t, p=p, omega=w)
    gR = torch.randn(2, 6, dtype=torch.complex128, generator=torch.Generator().manual_seed(0))
    ga = torch.autograd.grad(R, t["alpha"], gR, retain_graph=True)[0]
    _, J = _fake_compute(t["alpha"], t["beta"], t["rho"], t["thickness"], 0, 0, p, w, False, True)
    L = t["alpha"].shape[0]
    want = (gR.conj().unsqueeze(-2) * J).real.sum(-1).sum(0)[:L]
    assert torch.allclose(ga, want, rtol=1e-12, atol=1e-12)
    assert ("vjp", (2, 6)) in CALLS
    # create_graph=True: backward is itself differentiable in gR (Jacobian contraction)
    gR2 = gR.clone().requires_grad_(True)
    ga2 = torch.autograd.grad(R, t["alpha"], gR2, create_graph=True)[0]
    assert torch.allclose(ga2, want, rtol=1e-12, atol=1e-12)
    (d,) = torch.autograd.grad(ga2.sum(), gR2)
    assert torch.allclose(d, J[:, :L].sum(1), rtol=1e-12, atol=1e-12)


def test_jacrev_jacfwd_and_exact_hessians(fake):
    t = _model()
    w = torch.arange(1, 6, dtype=torch.float64) * 0.3
    m0 = KT._pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"])

    def f(m):
        a, b, r, h = KT._unpack_params(m, t["alpha"], t["beta"], t["rho"], t["thickness"])
        return KT.kennett_reflectivity_torch(a, b, r, h, t["Q_alpha"], t["Q_beta"], 0.3, w)

    full = KT._unpack_params(m0, t["alpha"], t["beta"], t["rho"], t["thickness"])
    R0, J = _fake_compute(*full, 0, 0, 0.3, w, False, True)
    L = t["alpha"].shape[0]
    idx = KT.packed_index(L)
    Jp = J[0][idx].T  # (nw, P)
    Jr = torch.func.jacrev(lambda m: f(m).real)(m0) + 1j * torch.func.jacrev(lambda m: f(m).imag)(m0)
    assert torch.allclose(Jr, Jp, rtol=1e-12, atol=1e-12)
    Jf = torch.func.jacfwd(lambda m: torch.view_as_real(f(m)))(m0)
    assert torch.allclose(Jf[..., 0, :] + 1j * Jf[..., 1, :], Jp, rtol=1e-12, atol=1e-12)
    R_obs = f(m0).detach() * 0.9

    def chi(m):
        r = f(m) - R_obs
        return (r.real**2 + r.imag**2).sum()

    # exact: 2 Re(J^H J) + 2 Re sum conj(res) d^2 R, with d^2 R / dm_a^2 = 2 c_a (diagonal)
    res = R0[0] - R_obs
    d2 = torch.stack([_fake_jacobian_dot(*full, 0, 0, 0.3, w, False,
                                         torch.eye(4 * L, dtype=torch.float64)[[i]])[0, 0, i]
                      for i in idx])  # (P, nw)
    H_exact = 2 * (Jp.conj().T @ Jp).real + torch.diag(2 * (res.conj() * d2).real.sum(-1))
    H = torch.func.hessian(chi)(m0)  # forward over reverse, as the reference takes it
    assert torch.allclose(H, H_exact, rtol=1e-10, atol=1e-10)
    assert not torch.allclose(H, 2 * (Jp.conj().T @ Jp).real, rtol=1e-6, atol=1e-6)
    # reverse over reverse through plain autograd (double backward)
    H2 = torch.autograd.functional.hessian(chi, m0)
    assert torch.allclose(H2, H_exact, rtol=1e-10, atol=1e-10)
    H3 = torch.func.jacrev(torch.func.jacrev(chi))(m0)
    assert torch.allclose(H3, H_exact, rtol=1e-10, atol=1e-10)
