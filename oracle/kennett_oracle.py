"""CPU oracle for the Kennett reflectivity path -- TEST INFRASTRUCTURE ONLY.

A NumPy/SciPy complex128 restatement of the reference algorithm
(tmnestor/SeismicInversion, ``Kennett_Reflectivity/``).  It is the checker the CUDA path is
compared against, and the CPU baseline that ``bench.py`` times.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs may import it;
the product package never does.

Parity pin: this restatement is checked against golden vectors produced by the reference
itself (``tests/golden/make_golden.py`` imports the reference and stores its outputs), see
``tests/test_oracle_golden.py``.

Every function keeps the reference's operation structure (full 2x2 complex matrices,
analytic inverse with four divisions, the same products in the same order) and is
vectorised over slowness *and* frequency instead of looping in Python.
"""

from __future__ import annotations

import numpy as np

__all__ = [
    "complex_slowness",
    "vertical_slowness",
    "solid_solid",
    "ocean_bottom",
    "reflectivity",
    "ricker_spectrum",
    "seismogram",
    "bessel_sum",
    "hermitian_traces",
    "gather",
    "fd_jacobian",
    "misfit",
]


def complex_slowness(v, Q):
    """s = (4Q^2 + 2iQ)/((1 + 4Q^2) v) -- ``layer_model.py:15-45`` (vectorised)."""
    v = np.asarray(v, dtype=np.float64)
    Q = np.asarray(Q, dtype=np.float64)
    twoQ = 2.0 * Q
    twoQsq = twoQ * twoQ
    den = (1.0 + twoQsq) * v
    return (twoQsq / den) + 1j * (twoQ / den)


def vertical_slowness(s, p):
    """eta = sqrt((s+p)(s-p)), negated where Im(eta) <= 0 -- ``layer_model.py:48-74``."""
    t = (s + p) * (s - p)
    eta = np.sqrt(t.astype(np.complex128))
    return np.where(eta.imag <= 0.0, -eta, eta)


def _layer_terms(alpha, beta, Qa, Qb):
    """Complex P/S slownesses and complex S velocity per layer (``layer_model.py:140-167``)."""
    s_p = complex_slowness(alpha, Qa)
    s_s = np.zeros(len(alpha), dtype=np.complex128)
    pos = beta > 0
    s_s[pos] = complex_slowness(beta[pos], Qb[pos])
    beta_c = np.zeros(len(alpha), dtype=np.complex128)
    nz = np.abs(s_s) > 0
    beta_c[nz] = 1.0 / s_s[nz]
    return s_p, s_s, beta_c


def solid_solid(p, eta1, neta1, rho1, beta1, eta2, neta2, rho2, beta2):
    """Modified P-SV coefficients at a solid-solid interface -- ``scattering_matrices.py:42-161``.

    ``p``/``eta*``/``neta*`` are arrays over slowness; returns (Rd, Ru, Tu, Td) of shape
    ``(np, 2, 2)``.
    """
    rtrho1 = np.sqrt(rho1)
    rtrho2 = np.sqrt(rho2)
    rteta1 = np.sqrt(eta1)
    rteta2 = np.sqrt(eta2)
    rtneta1 = np.sqrt(neta1)
    rtneta2 = np.sqrt(neta2)
    rtza1 = rteta1 * rtrho1
    rtza2 = rteta2 * rtrho2
    rtzb1 = rtneta1 * rtrho1
    rtzb2 = rtneta2 * rtrho2
    psq = (p * p).astype(np.complex128)
    crho1 = complex(rho1)
    crho2 = complex(rho2)
    drho = crho2 - crho1
    dmu = crho2 * beta2 * beta2 - crho1 * beta1 * beta1
    d = 2.0 * dmu
    psqd = psq * d
    a = drho - psqd
    b = crho2 - psqd
    c = crho1 + psqd
    E = b * eta1 + c * eta2
    F = b * neta1 + c * neta2
    G = a - d * eta1 * neta2
    H = a - d * eta2 * neta1
    Det = E * F + G * H * psq
    E = E / Det
    F = F / Det
    G = G / Det
    H = H / Det
    Qv = (b * eta1 - c * eta2) * F
    Rv = (a + d * eta1 * neta2) * H * psq
    Sv = (a * b + c * d * eta2 * neta2) * p / Det
    Tv = (b * neta1 - c * neta2) * E
    Uv = (a + d * eta2 * neta1) * G * psq
    Vv = (a * c + b * d * eta1 * neta1) * p / Det
    m2ci = complex(0.0, -2.0)
    n = len(p)
    Rd = np.empty((n, 2, 2), dtype=np.complex128)
    Rd[:, 0, 0] = Qv - Rv
    Rd[:, 0, 1] = m2ci * rteta1 * rtneta1 * Sv
    Rd[:, 1, 0] = m2ci * rteta1 * rtneta1 * Sv
    Rd[:, 1, 1] = Tv - Uv
    Td = np.empty((n, 2, 2), dtype=np.complex128)
    Td[:, 0, 0] = 2 * rtza1 * rtza2 * F
    Td[:, 0, 1] = m2ci * rtzb1 * rtza2 * G * p
    Td[:, 1, 0] = m2ci * rtza1 * rtzb2 * H * p
    Td[:, 1, 1] = 2 * rtzb1 * rtzb2 * E
    Tu = np.transpose(Td, (0, 2, 1)).copy()
    Ru = np.empty((n, 2, 2), dtype=np.complex128)
    Ru[:, 0, 0] = -(Qv + Uv)
    Ru[:, 0, 1] = m2ci * rteta2 * rtneta2 * Vv
    Ru[:, 1, 0] = m2ci * rteta2 * rtneta2 * Vv
    Ru[:, 1, 1] = -(Tv + Rv)
    return Rd, Ru, Tu, Td


def ocean_bottom(p, eta1, rho1, eta2, neta2, rho2, beta2):
    """Acoustic-elastic (ocean-bottom) coefficients -- ``scattering_matrices.py:164-296``."""
    rtrho1 = np.sqrt(rho1)
    rtrho2 = np.sqrt(rho2)
    rteta1 = np.sqrt(eta1)
    rteta2 = np.sqrt(eta2)
    rtneta2 = np.sqrt(neta2)
    rtza1 = rtrho1 * rteta1
    rtza2 = rtrho2 * rteta2
    rtzb2 = rtrho2 * rtneta2
    psq = p * p
    crho1 = complex(rho1)
    crho2 = complex(rho2)
    drho = crho2 - crho1
    dmu = crho2 * beta2 * beta2
    d = 2.0 * dmu
    psqd = psq * d
    a = drho - psqd
    b = crho2 - psqd
    c = crho1 + psqd
    E = b * eta1 + c * eta2
    F = b
    G = a - d * eta1 * neta2
    H = -d * eta2
    Det = E * F + G * H * psq
    E = E / Det
    F = F / Det
    G = G / Det
    H = H / Det
    T1 = (b * eta1 - c * eta2) * F
    T2 = (a + d * eta1 * neta2) * H * psq
    T4 = b * E
    T5 = d * eta2 * G * psq
    T6 = b * d * eta1 * p / Det
    mci = complex(0.0, -1.0)
    n = len(p)
    z = np.zeros(n, dtype=np.complex128)
    PdPd = 2.0 * rtza1 * rtza2 * F
    PdSd = 2.0 * mci * rtza1 * rtzb2 * H * p
    PuSd = 2.0 * mci * rteta2 * rtneta2 * T6
    Rd = np.stack([np.stack([T1 - T2, z], -1), np.stack([z, z], -1)], -2)
    Td = np.stack([np.stack([PdPd, z], -1), np.stack([PdSd, z], -1)], -2)
    Tu = np.stack([np.stack([PdPd, PdSd], -1), np.stack([z, z], -1)], -2)
    Ru = np.stack([np.stack([-(T1 + T5), PuSd], -1), np.stack([PuSd, -(T2 + T4)], -1)], -2)
    return Rd, Ru, Tu, Td


def _is_half_space(h):
    return np.isinf(h) or h >= 1e30


def _inv2x2(M):
    """Analytic 2x2 inverse with four divisions -- ``kennett_reflectivity.py:29-51``."""
    a = M[..., 0, 0]
    b = M[..., 0, 1]
    c = M[..., 1, 0]
    d = M[..., 1, 1]
    det = a * d - b * c
    inv = np.empty_like(M)
    inv[..., 0, 0] = d / det
    inv[..., 0, 1] = -b / det
    inv[..., 1, 0] = -c / det
    inv[..., 1, 1] = a / det
    return inv


def reflectivity(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface=False):
    """R(p, omega) for an array of slownesses -- ``kennett_reflectivity.py:73-328``.

    ``p``: float array ``(np,)``; ``omega``: real or complex ``(nw,)``.  Returns complex128
    ``(np, nw)``.  Upward sweep from the half-space with RRd = 0; per interface
    MT = E RRd E, U = (I - Ru MT)^-1, RRd = Rd + Tu MT U Td; then the ocean two-way phase
    and, with ``free_surface``, R = E^2 RRd_PP / (1 + E^2 RRd_PP).
    """
    alpha, beta, rho, thickness, Q_alpha, Q_beta = (
        np.asarray(x, dtype=np.float64) for x in (alpha, beta, rho, thickness, Q_alpha, Q_beta)
    )
    p = np.atleast_1d(np.asarray(p, dtype=np.float64))
    omega = np.asarray(omega)
    L = len(alpha)
    npp = len(p)
    nw = len(omega)
    s_p, s_s, beta_c = _layer_terms(alpha, beta, Q_alpha, Q_beta)
    cp = p.astype(np.complex128)
    eta = vertical_slowness(s_p[:, None], cp[None, :])  # (L, np)
    neta = vertical_slowness(s_s[:, None], cp[None, :])
    neta[0] = 0.0

    def phases(i):
        if _is_half_space(thickness[i]):
            one = np.ones((npp, nw), dtype=np.complex128)
            return one, one
        ea = np.exp(1j * omega[None, :] * eta[i][:, None] * thickness[i])
        eb = np.exp(1j * omega[None, :] * neta[i][:, None] * thickness[i])
        return ea, eb

    scat = [ocean_bottom(p, eta[0], rho[0], eta[1], neta[1], rho[1], beta_c[1])]
    for il in range(1, L - 1):
        scat.append(
            solid_solid(p, eta[il], neta[il], rho[il], beta_c[il],
                        eta[il + 1], neta[il + 1], rho[il + 1], beta_c[il + 1])
        )
    RRd = np.zeros((npp, nw, 2, 2), dtype=np.complex128)
    eye = np.eye(2, dtype=np.complex128)
    for iface in range(L - 2, -1, -1):
        Rd, Ru, Tu, Td = scat[iface]
        ea, eb = phases(iface + 1)
        eaea = ea**2
        ebeb = eb**2
        eaeb = ea * eb
        MT = np.empty_like(RRd)
        MT[..., 0, 0] = eaea * RRd[..., 0, 0]
        MT[..., 0, 1] = eaeb * RRd[..., 0, 1]
        MT[..., 1, 0] = eaeb * RRd[..., 1, 0]
        MT[..., 1, 1] = ebeb * RRd[..., 1, 1]
        RuMT = np.einsum("pij,pwjk->pwik", Ru, MT)
        U = _inv2x2(eye - RuMT)
        MTU = np.einsum("pwij,pwjk->pwik", MT, U)
        TuMTU = np.einsum("pij,pwjk->pwik", Tu, MTU)
        RRd = Rd[:, None] + np.einsum("pwij,pjk->pwik", TuMTU, Td)
    rpp = RRd[..., 0, 0]
    ea0, _ = phases(0)
    e2 = ea0**2
    if not free_surface:
        return e2 * rpp
    return (e2 * rpp) / (1.0 + e2 * rpp)


def ricker_spectrum(omega, omega_max):
    """``source.py:10-45``."""
    a = 0.1 * omega_max
    t0 = 5.0 / (a * np.sqrt(2.0))
    z = (omega**2) / (4.0 * a**2)
    return z * np.exp(-z + 1j * omega * t0)


def hermitian_traces(Y, nw, decay=None):
    """Real traces from positive-frequency spectra -- ``kennett_seismogram.py:124-144``.

    ``Y``: ``(..., nw-1)`` values at omega_1..omega_{nw-1}.  Builds the length-2nw Hermitian
    spectrum (DC and Nyquist zero), applies the *forward* DFT and keeps the real part,
    times ``decay`` (e.g. exp(-gamma t)) if given.
    """
    Y = np.atleast_2d(Y)
    nt = 2 * nw
    X = np.zeros(Y.shape[:-1] + (nt,), dtype=np.complex128)
    X[..., 1:nw] = Y
    X[..., nw + 1:] = np.conj(Y[..., ::-1])
    out = np.real(np.fft.fft(X, axis=-1))
    if decay is not None:
        out = out * decay
    return out


def seismogram(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, T=64.0, nw=2048, eps=0.0,
               source=None, free_surface=False):
    """Single-slowness trace -- ``kennett_seismogram.py:57-150``.  ``source(omega, wmax)``."""
    dw = 2.0 * np.pi / T
    omega = np.arange(1, nw, dtype=np.float64) * dw
    wmax = nw * dw
    S = ricker_spectrum(omega, wmax) if source is None else source(omega, wmax)
    R = reflectivity(alpha, beta, rho, thickness, Q_alpha, Q_beta, [p], omega, free_surface)[0]
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    trace = hermitian_traces(R * S, nw)[0] * np.exp(eps * time)
    return time, trace, R


def bessel_sum(R, p_samples, omega_real, offsets, dp, taper=None, chunk=64):
    """U(r, w) = sum_j R[j, w] taper_j p_j w dp J0(w p_j r) in float64.

    Follows ``kennett_gather.py:112-124`` (per-slowness contribution, argument formed as
    (w p_j) r, weight ((taper_j p_j) w) dp), summed in slowness order.
    """
    from scipy.special import j0

    R = np.asarray(R)
    p_samples = np.asarray(p_samples, dtype=np.float64)
    omega_real = np.asarray(omega_real, dtype=np.float64)
    offsets = np.asarray(offsets, dtype=np.float64)
    U = np.zeros((len(offsets), len(omega_real)), dtype=np.complex128)
    for j0_ in range(0, len(p_samples), chunk):
        sl = slice(j0_, min(j0_ + chunk, len(p_samples)))
        pj = p_samples[sl]
        arg = (omega_real[None, None, :] * pj[:, None, None]) * offsets[None, :, None]
        J = j0(arg)  # (c, nr, nw)
        tap = taper[sl] if taper is not None else np.ones(len(pj))
        w = ((tap * pj)[:, None] * omega_real[None, :]) * dp  # (c, nw)
        U += np.einsum("crw,cw->rw", J, R[sl] * w)
    return U


def gather(alpha, beta, rho, thickness, Q_alpha, Q_beta, offsets, T=64.0, nw=2048,
           np_slow=2048, p_max=1.0, gamma=None, source=None, free_surface=False, p_chunk=32):
    """Discrete-wavenumber gather -- ``kennett_gather.py:127-305`` (float64 throughout).

    Returns ``(time, offsets, gather, R)`` with ``R`` the (np, nw-1) reflectivity grid at
    the damped frequencies.
    """
    if gamma is None:
        gamma = np.pi / T
    dw = 2.0 * np.pi / T
    omega = np.arange(1, nw, dtype=np.float64) * dw
    wmax = nw * dw
    S = ricker_spectrum(omega, wmax) if source is None else source(omega, wmax)
    dp = p_max / np_slow
    p = np.arange(1, np_slow + 1, dtype=np.float64) * dp
    taper = 0.5 * (1.0 + np.cos(np.pi * p / p_max))
    R = np.empty((np_slow, nw - 1), dtype=np.complex128)
    for k in range(0, np_slow, p_chunk):
        R[k:k + p_chunk] = reflectivity(alpha, beta, rho, thickness, Q_alpha, Q_beta,
                                        p[k:k + p_chunk], omega + 1j * gamma, free_surface)
    U = bessel_sum(R, p, omega, offsets, dp, taper)
    U *= S[None, :]
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    g = hermitian_traces(U, nw, np.exp(-gamma * time))
    return time, np.asarray(offsets), g, R


def misfit(R, R_obs):
    """chi = sum |R - R_obs|^2 (``taup_inversion.py:106-107``)."""
    r = R - R_obs
    return float(np.sum(r.real**2 + r.imag**2))


def fd_jacobian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface=False,
                delta=1e-7, params=None):
    """Central finite-difference dR/dm over the reference's packed sub-ocean parameters.

    Parameter order ``[Vp_1..N, Vs_1..N, rho_1..N, h_1..N-1]`` (``kennett_torch.py:552-571``);
    ``params`` may select a subset of indices.  Same scheme as
    ``test_torch_gradients.py:153-186`` (delta = 1e-7, absolute step).  Returns
    ``(np, nw, P)``.
    """
    base = [np.asarray(x, dtype=np.float64).copy() for x in (alpha, beta, rho, thickness)]
    L = len(base[0])
    n_sub = L - 1
    idx = []
    for k in range(n_sub):
        idx.append((0, k + 1))
    for k in range(n_sub):
        idx.append((1, k + 1))
    for k in range(n_sub):
        idx.append((2, k + 1))
    for k in range(n_sub - 1):
        idx.append((3, k + 1))
    sel = range(len(idx)) if params is None else params
    p = np.atleast_1d(p)
    out = np.zeros((len(p), len(omega), len(list(sel))), dtype=np.complex128)
    for col, j in enumerate(sel):
        arr, layer = idx[j]
        res = []
        for sgn in (1.0, -1.0):
            m = [b.copy() for b in base]
            m[arr][layer] += sgn * delta
            res.append(reflectivity(*m, Q_alpha, Q_beta, p, omega, free_surface))
        out[:, :, col] = (res[0] - res[1]) / (2.0 * delta)
    return out
