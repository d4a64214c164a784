"""Host logic of the finite-difference Hessians (``_Problem.stencil_rows`` /
``stencil_hessian``): against an analytic gradient, the second-order stencil is accurate to
O(d^2) and the fourth-order one to O(d^4), with the perturbed rows laid out as the batched
launch expects (block k moves every parameter by offset k times its own step)."""

import numpy as np
import pytest

from seismicinversion_b200.taup_inversion import _Problem


def _grad(m, A):
    # gradient of f(m) = m^T A m / 2 + sum exp(0.3 m) m^2 / 10
    return A @ m + (0.03 * np.exp(0.3 * m) * m**2 + 0.2 * np.exp(0.3 * m) * m) / 1.0


def _hess(m, A):
    e = np.exp(0.3 * m)
    return A + np.diag(0.009 * e * m**2 + 0.06 * e * m + 0.06 * e * m + 0.2 * e)


@pytest.mark.parametrize("stencil,tol", [(2, 1e-7), (4, 1e-10)])
def test_stencils_against_analytic_hessian(stencil, tol):
    rng = np.random.default_rng(1)
    P = 9
    B = rng.standard_normal((P, P))
    A = B @ B.T
    m = rng.uniform(0.5, 3.0, P)
    rows, d = _Problem.stencil_rows(m, 1e-5, stencil)
    K = len(_Problem._STENCILS[stencil][0])
    assert rows.shape == (K * P, P)
    # every row differs from m in exactly one parameter
    diff = rows - m[None, :]
    assert np.all(np.count_nonzero(diff, axis=1) == 1)
    g = np.stack([_grad(r, A) for r in rows])
    H = _Problem.stencil_hessian(g, d, stencil)
    ref = _hess(m, A)
    assert np.abs(H - ref).max() / np.abs(ref).max() < tol
    assert np.array_equal(H, H.T)


def test_fourth_order_beats_second_order():
    rng = np.random.default_rng(2)
    P = 6
    A = np.diag(rng.uniform(1, 2, P))
    m = rng.uniform(0.5, 3.0, P)
    errs = []
    for stencil in (2, 4):
        rows, d = _Problem.stencil_rows(m, 1e-3, stencil)
        H = _Problem.stencil_hessian(np.stack([_grad(r, A) for r in rows]), d, stencil)
        errs.append(np.abs(H - _hess(m, A)).max())
    assert errs[1] < 1e-3 * errs[0]


class _FakeProblem:
    """chi(m) = sum_i c_i m_i^3 with analytic gradient and Hessian (physical parameters)."""

    def __init__(self, c):
        self.c = c

    def chi_grad(self, m):
        return float(np.sum(self.c * m**3)), 3 * self.c * m**2

    def hessian_exact(self, m):
        return np.diag(6 * self.c * m)

    hessian_gn = hessian_exact


def test_log_space_gradient_and_hessian():
    """taup_misfit_grad_hessian's chain rule to log parameters (taup_inversion.py:183-185):
    g_log = m g and H_log = m m^T H + diag(g m), against the derivatives of chi(exp(x))."""
    from seismicinversion_b200.taup_inversion import _chi_g_h, newton_lm_step

    rng = np.random.default_rng(3)
    c = rng.uniform(0.5, 2.0, 5)
    x = rng.uniform(-0.5, 0.5, 5)
    chi, g_log, H_log = _chi_g_h(_FakeProblem(c), x, "exact")
    m = np.exp(x)
    assert chi == pytest.approx(np.sum(c * m**3))
    assert np.allclose(g_log, 3 * c * m**3)            # d/dx c e^{3x} = 3 c e^{3x}
    assert np.allclose(H_log, np.diag(9 * c * m**3))   # d2/dx2 = 9 c e^{3x}
    with pytest.raises(ValueError):
        _chi_g_h(_FakeProblem(c), x, "newton")
    dx = newton_lm_step(g_log, H_log, 0.1)
    assert np.allclose((H_log + 0.1 * np.eye(5)) @ dx, -g_log)
