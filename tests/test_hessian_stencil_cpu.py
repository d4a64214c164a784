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
