"""Differentiable CPU oracle of the Kennett reflectivity -- TEST / BENCH INFRASTRUCTURE ONLY.

A torch (complex128, CPU) restatement of the reference's differentiable forward
``kennett_reflectivity_torch`` (tmnestor/SeismicInversion,
``Kennett_Reflectivity/kennett_torch.py:312-480``), with the operation structure of the
NumPy oracle (``oracle/kennett_oracle.py``: full 2x2 matrices, analytic inverse with four
divisions), vectorised over slowness and frequency and written without in-place updates so
that torch autograd differentiates it: gradients by ``torch.autograd.grad`` as the
reference's ``taup_misfit_grad_hessian`` takes them (``taup_inversion.py:153-172``),
Jacobians by ``torch.func.jacrev`` (``kennett_torch.py:611-641``), Hessians by
``torch.func.hessian`` (``:644-684``).  It is the CPU baseline of the tau-p derivative
workloads in ``bench.py`` and a cross-check of the derivative goldens.

Parity pin: ``tests/test_oracle_golden.py`` checks it against the NumPy oracle and against
the reference's own jacrev / autograd goldens (``tests/golden/derivs_c2_1024.npz``,
``derivs_default.npz``).  Only ``tests/`` and ``bench.py``'s CPU-baseline legs import it.
"""

from __future__ import annotations

import torch

_C = torch.complex128
_F = torch.float64

__all__ = ["reflectivity", "misfit"]


def _cslow(v, Q):
    """s = (4Q^2 + 2iQ)/((1 + 4Q^2) v) -- ``layer_model.py:15-45``."""
    twoQ = 2.0 * Q
    twoQsq = twoQ * twoQ
    den = (1.0 + twoQsq) * v
    return torch.complex(twoQsq / den, twoQ / den)


def _vslow(s, p):
    """eta = sqrt((s+p)(s-p)), negated where Im(eta) <= 0 -- ``layer_model.py:48-74``."""
    eta = torch.sqrt((s + p) * (s - p))
    return torch.where(eta.imag <= 0.0, -eta, eta)


def _m22(a, b, c, d):
    return torch.stack([torch.stack([a, b], -1), torch.stack([c, d], -1)], -2)


def _solid_solid(p, eta1, neta1, rho1, beta1, eta2, neta2, rho2, beta2):
    """``scattering_matrices.py:42-161`` over slowness: (Rd, Ru, Tu, Td), each (np, 2, 2)."""
    rtrho1, rtrho2 = torch.sqrt(rho1.to(_C)), torch.sqrt(rho2.to(_C))
    rteta1, rteta2 = torch.sqrt(eta1), torch.sqrt(eta2)
    rtneta1, rtneta2 = torch.sqrt(neta1), torch.sqrt(neta2)
    rtza1, rtza2 = rteta1 * rtrho1, rteta2 * rtrho2
    rtzb1, rtzb2 = rtneta1 * rtrho1, rtneta2 * rtrho2
    psq = (p * p).to(_C)
    crho1, crho2 = rho1.to(_C), rho2.to(_C)
    dmu = crho2 * beta2 * beta2 - crho1 * beta1 * beta1
    d = 2.0 * dmu
    psqd = psq * d
    a = (crho2 - crho1) - psqd
    b = crho2 - psqd
    c = crho1 + psqd
    E = b * eta1 + c * eta2
    F = b * neta1 + c * neta2
    G = a - d * eta1 * neta2
    H = a - d * eta2 * neta1
    Det = E * F + G * H * psq
    E, F, G, H = E / Det, F / Det, G / Det, H / Det
    Qv = (b * eta1 - c * eta2) * F
    Rv = (a + d * eta1 * neta2) * H * psq
    Sv = (a * b + c * d * eta2 * neta2) * p / Det
    Tv = (b * neta1 - c * neta2) * E
    Uv = (a + d * eta2 * neta1) * G * psq
    Vv = (a * c + b * d * eta1 * neta1) * p / Det
    m2i = complex(0.0, -2.0)
    rd12 = m2i * rteta1 * rtneta1 * Sv
    ru12 = m2i * rteta2 * rtneta2 * Vv
    Rd = _m22(Qv - Rv, rd12, rd12, Tv - Uv)
    Td = _m22(2 * rtza1 * rtza2 * F, m2i * rtzb1 * rtza2 * G * p,
              m2i * rtza1 * rtzb2 * H * p, 2 * rtzb1 * rtzb2 * E)
    Ru = _m22(-(Qv + Uv), ru12, ru12, -(Tv + Rv))
    return Rd, Ru, Td.transpose(-1, -2), Td


def _ocean_bottom(p, eta1, rho1, eta2, neta2, rho2, beta2):
    """``scattering_matrices.py:164-296`` over slowness."""
    rtrho1, rtrho2 = torch.sqrt(rho1.to(_C)), torch.sqrt(rho2.to(_C))
    rteta1, rteta2, rtneta2 = torch.sqrt(eta1), torch.sqrt(eta2), torch.sqrt(neta2)
    rtza1, rtza2, rtzb2 = rtrho1 * rteta1, rtrho2 * rteta2, rtrho2 * rtneta2
    psq = (p * p).to(_C)
    crho1, crho2 = rho1.to(_C), rho2.to(_C)
    d = 2.0 * (crho2 * beta2 * beta2)
    psqd = psq * d
    a = (crho2 - crho1) - psqd
    b = crho2 - psqd
    c = crho1 + psqd
    E = b * eta1 + c * eta2
    F = b
    G = a - d * eta1 * neta2
    H = -d * eta2
    Det = E * F + G * H * psq
    E, F, G, H = E / Det, F / Det, G / Det, H / Det
    T1 = (b * eta1 - c * eta2) * F
    T2 = (a + d * eta1 * neta2) * H * psq
    T4 = b * E
    T5 = d * eta2 * G * psq
    T6 = b * d * eta1 * p / Det
    mci = complex(0.0, -1.0)
    z = torch.zeros_like(T1)
    PdPd = 2.0 * rtza1 * rtza2 * F
    PdSd = 2.0 * mci * rtza1 * rtzb2 * H * p
    PuSd = 2.0 * mci * rteta2 * rtneta2 * T6
    Rd = _m22(T1 - T2, z, z, z)
    Td = _m22(PdPd, z, PdSd, z)
    Tu = _m22(PdPd, PdSd, z, z)
    Ru = _m22(-(T1 + T5), PuSd, PuSd, -(T2 + T4))
    return Rd, Ru, Tu, Td


def _inv2x2(M):
    """Analytic inverse with four divisions -- ``kennett_reflectivity.py:29-51``."""
    a, b, c, d = M[..., 0, 0], M[..., 0, 1], M[..., 1, 0], M[..., 1, 1]
    det = a * d - b * c
    return _m22(d / det, -b / det, -c / det, a / det)


def reflectivity(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface=False):
    """R(p, omega), complex128 (np, nw), differentiable in alpha, beta, rho, thickness.

    The half-space is the last layer (its thickness, +inf or >= 1e30, never enters: phase 1);
    derivatives through the ocean's S quantities and the half-space phase are zero, as the
    reference's torch.where masks give."""
    L = alpha.shape[0]
    p = torch.as_tensor(p, dtype=_F).reshape(-1)
    omega = torch.as_tensor(omega).to(_C).reshape(-1)
    cp = p.to(_C)
    s_p = _cslow(alpha, Q_alpha)
    pos = beta > 0
    b_safe = torch.where(pos, beta, torch.ones_like(beta))
    s_s = torch.where(pos, _cslow(b_safe, Q_beta), torch.zeros((), dtype=_C))
    s_s_safe = torch.where(pos, s_s, torch.ones((), dtype=_C))
    beta_c = torch.where(pos, 1.0 / s_s_safe, torch.zeros((), dtype=_C))
    eta = _vslow(s_p[:, None], cp[None, :])  # (L, np)
    neta_all = _vslow(s_s_safe[:, None], cp[None, :])
    neta = torch.cat([torch.zeros_like(neta_all[:1]), torch.where(pos[1:, None], neta_all[1:],
                                                                   torch.zeros((), dtype=_C))])

    def phases(i):
        h = float(thickness[i].detach())
        if h == float("inf") or h >= 1e30:
            one = torch.ones((len(p), len(omega)), dtype=_C)
            return one, one
        hh = thickness[i].to(_C)
        ea = torch.exp(1j * omega[None, :] * eta[i][:, None] * hh)
        eb = torch.exp(1j * omega[None, :] * neta[i][:, None] * hh)
        return ea, eb

    scat = [_ocean_bottom(p, eta[0], rho[0], eta[1], neta[1], rho[1], beta_c[1])]
    for il in range(1, L - 1):
        scat.append(_solid_solid(p, eta[il], neta[il], rho[il], beta_c[il], eta[il + 1],
                                 neta[il + 1], rho[il + 1], beta_c[il + 1]))
    RRd = torch.zeros((len(p), len(omega), 2, 2), dtype=_C)
    eye = torch.eye(2, dtype=_C)
    for iface in range(L - 2, -1, -1):
        Rd, Ru, Tu, Td = scat[iface]
        ea, eb = phases(iface + 1)
        MT = _m22(ea * ea * RRd[..., 0, 0], ea * eb * RRd[..., 0, 1], ea * eb * RRd[..., 1, 0],
                  eb * eb * RRd[..., 1, 1])
        U = _inv2x2(eye - torch.einsum("pij,pwjk->pwik", Ru, MT))
        TuMTU = torch.einsum("pij,pwjk->pwik", Tu, torch.einsum("pwij,pwjk->pwik", MT, U))
        RRd = Rd[:, None] + torch.einsum("pwij,pjk->pwik", TuMTU, Td)
    ea0, _ = phases(0)
    y = ea0 * ea0 * RRd[..., 0, 0]
    return y / (1.0 + y) if free_surface else y


def misfit(R, R_obs):
    """chi = sum |R - R_obs|^2."""
    r = R - R_obs
    return (r.real ** 2 + r.imag ** 2).sum()
