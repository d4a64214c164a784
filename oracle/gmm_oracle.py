"""CPU oracle for the Global Matrix Method reflectivity -- TEST INFRASTRUCTURE ONLY.

A NumPy complex128 restatement of the reference's block-Riccati GMM forward
(tmnestor/SeismicInversion, ``GlobalMatrix/``), vectorised over slowness and frequency.
Only ``tests/`` may import it; the product package never does.

Parity pin: checked against golden vectors produced by the reference's own
``global_matrix.gmm_reflectivity`` and ``gmm_torch.gmm_reflectivity_torch``
(``tests/golden/make_golden.py --gmm-only``), see ``tests/test_oracle_golden.py``.

Steps, each citing the reference:
  layer eigenvectors    ``layer_matrix.py:24-95``  (E_d, E_u 4x2; ocean e_d, e_u)
  phases                ``global_matrix.py:24-63`` (exp(i w eta h), exp(i w neta h), e0)
  Riccati sweep         ``riccati_solver.py:25-126`` (E_eff = E_d + E_u diag(ph) Y,
                        F = [E_u | -E_eff], F X = -E_d diag(ph), Y = X[:2])
  ocean extraction      ``riccati_solver.py:141-198``
  free surface          ``global_matrix.py:345-346`` (R / (1 + R))
The 4x4 systems are solved with ``numpy.linalg.solve`` (LAPACK gesv, partial pivoting), as
the reference does.
"""

from __future__ import annotations

import numpy as np

from .kennett_oracle import _layer_terms, vertical_slowness

__all__ = ["gmm_reflectivity"]


def _eigenvectors(p, eta, neta, rho, beta_c):
    """E_d, E_u with shape (..., 4, 2) for broadcast arrays of layer terms."""
    cp = np.asarray(p, dtype=np.complex128)
    crho = np.asarray(rho, dtype=np.complex128)
    mu = crho * beta_c * beta_c
    gamma = crho * (1.0 - 2.0 * beta_c * beta_c * cp * cp)
    a = 2.0 * mu * cp * neta
    b = 2.0 * mu * cp * eta
    cp = np.broadcast_to(cp, eta.shape)
    E_d = np.stack([np.stack([cp, neta], -1), np.stack([eta, -cp], -1),
                    np.stack([-gamma, a], -1), np.stack([b, gamma], -1)], -2)
    E_u = np.stack([np.stack([cp, -neta], -1), np.stack([-eta, -cp], -1),
                    np.stack([-gamma, -a], -1), np.stack([-b, gamma], -1)], -2)
    return E_d, E_u


def gmm_reflectivity(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                     free_surface=False):
    """R(p, omega) by the block-Riccati Global Matrix Method; returns complex128 (np, nw)."""
    alpha, beta, rho, thickness, Q_alpha, Q_beta = (
        np.asarray(x, dtype=np.float64) for x in (alpha, beta, rho, thickness, Q_alpha, Q_beta)
    )
    p = np.atleast_1d(np.asarray(p, dtype=np.float64))
    omega = np.asarray(omega).astype(np.complex128)
    L = len(alpha)
    s_p, s_s, beta_c = _layer_terms(alpha, beta, Q_alpha, Q_beta)
    cp = p.astype(np.complex128)
    eta = vertical_slowness(s_p[:, None], cp[None, :])  # (L, np)
    neta = vertical_slowness(s_s[:, None], cp[None, :])
    neta[0] = 0.0
    # (L, np, 4, 2) eigenvectors; phases (L, np, nw, 2)
    E_d, E_u = _eigenvectors(cp[None, :], eta, neta, rho[:, None], beta_c[:, None])
    e0 = np.exp(1j * omega[None, :] * eta[0][:, None] * thickness[0])  # (np, nw)
    ph = np.ones((L, len(p), len(omega), 2), dtype=np.complex128)
    for j in range(1, L - 1):
        ph[j, :, :, 0] = np.exp(1j * omega[None, :] * eta[j][:, None] * thickness[j])
        ph[j, :, :, 1] = np.exp(1j * omega[None, :] * neta[j][:, None] * thickness[j])
    M = L - 2
    shape = (len(p), len(omega))
    Y = np.zeros(shape + (2, 2), dtype=np.complex128)
    for k in range(M, 0, -1):
        kb = k + 1
        if kb < L - 1:
            Eu_ph = E_u[kb][:, None, :, :] * ph[kb][:, :, None, :]
            E_eff = E_d[kb][:, None, :, :] + Eu_ph @ Y
        else:
            E_eff = np.broadcast_to(E_d[kb][:, None, :, :], shape + (4, 2))
        A_d = E_d[k][:, None, :, :] * ph[k][:, :, None, :]
        F = np.concatenate([np.broadcast_to(E_u[k][:, None, :, :], shape + (4, 2)), -E_eff],
                           axis=-1)
        X = np.linalg.solve(F, -A_d)
        Y = X[..., :2, :]
    if M >= 1:
        E1 = E_d[1][:, None, :, :] + (E_u[1][:, None, :, :] * ph[1][:, :, None, :]) @ Y
    else:
        E1 = np.broadcast_to(E_d[1][:, None, :, :], shape + (4, 2))
    # ocean eigenvectors e_d = (eta0, -rho0), e_u = (-eta0, -rho0)
    eta0 = eta[0][:, None]
    ed = (eta0, -rho[0] + 0j)
    eu = (-eta0, -rho[0] + 0j)
    row_A = eu[0][..., None] * E1[..., 2, :] - eu[1] * E1[..., 1, :]
    row_B = E1[..., 3, :]
    mat = np.stack([row_A, row_B], axis=-2)
    rhs = np.stack([(eu[0] * ed[1] - eu[1] * ed[0]) * e0, np.zeros(shape, np.complex128)], -1)
    D1 = np.linalg.solve(mat, rhs[..., None])[..., 0]
    uz = np.sum(E1[..., 1, :] * D1, axis=-1)
    U0 = (uz - ed[0] * e0) / eu[0]
    R = e0 * U0
    if free_surface:
        R = R / (1.0 + R)
    return R
