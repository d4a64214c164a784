"""Drop-in for the compute part of ``Kennett_Reflectivity.taup_inversion`` (``taup_inversion.py:56-571``).

Same Newton / Levenberg-Marquardt scheme in log-parameter space (``invert_taup``:
lambda0 = 0.01 max|diag H|, accept -> lambda / 2, reject -> lambda * 5, <= 10 trials,
``taup_inversion.py:389-439``) and the same log transform of gradient and Hessian
(``:183-185``).  What changes is where the numbers come from: the misfit and gradient over
all slownesses are one launch of the adjoint kernel (``kr_misfit_gradient``) instead of a
per-slowness autograd pass, and the Hessian is either

* ``hessian="exact"`` (default): the exact Hessian, as the reference's
  ``torch.func.hessian`` gives it, from one launch of the tangent-of-adjoint kernel
  (``kr_misfit_hvp``: H e_j for every packed parameter j, no step size); or
* ``hessian="gauss-newton"``: 2 Re(J^H J) from one ``kr_jacobian`` launch.

The LaTeX / TikZ / plotting writers of the reference module are presentation, not compute,
and are not mirrored.
"""

from __future__ import annotations

import logging
from dataclasses import dataclass, field

import numpy as np
import torch

from . import device as D
from .kennett_torch import _pack_params, _unpack_params, model_to_tensors, packed_index
from .layer_model import LayerModel
from .source import ricker_spectrum

__all__ = [
    "InversionResult",
    "taup_misfit_grad_hessian",
    "newton_lm_step",
    "invert_taup",
    "compute_taup_traces",
]

logger = logging.getLogger(__name__)
_FDTYPE = torch.float64


@dataclass
class InversionResult:
    """Convergence history and models (``taup_inversion.py:56-67``)."""

    true_model: LayerModel
    initial_model: LayerModel
    recovered_model: LayerModel
    misfit_history: list = field(default_factory=list)
    grad_norm_history: list = field(default_factory=list)
    param_error_history: list = field(default_factory=list)
    n_iterations: int = 0
    converged: bool = False


def _obs_matrix(R_obs, p_values, dev) -> torch.Tensor:
    if isinstance(R_obs, dict):
        rows = [torch.as_tensor(R_obs[p]) for p in p_values]
        return torch.stack(rows).to(dev, torch.complex128)
    return torch.as_tensor(R_obs).to(dev, torch.complex128).reshape(len(p_values), -1)


class _Problem:
    """Fixed data of one tau-p inversion, resident on the device."""

    def __init__(self, alpha_ref, beta_ref, rho_ref, thickness_ref, Q_alpha, Q_beta, p_values,
                 omega, R_obs, free_surface: bool = False):
        self.dev = D.require_cuda()
        self.fs = bool(free_surface)
        self.ref = [torch.as_tensor(x, dtype=_FDTYPE).detach().cpu()
                    for x in (alpha_ref, beta_ref, rho_ref, thickness_ref)]
        self.Q = [torch.as_tensor(x, dtype=_FDTYPE).detach().cpu() for x in (Q_alpha, Q_beta)]
        self.p = torch.as_tensor(np.asarray(p_values, dtype=np.float64), device=self.dev)
        self.omega = torch.as_tensor(omega).detach().to(self.dev, torch.complex128)
        self.R_obs = _obs_matrix(R_obs, list(p_values), self.dev)
        self.L = self.ref[0].shape[0]
        self.idx = packed_index(self.L)

    def table(self, phys: np.ndarray) -> torch.Tensor:
        a, b, r, h = _unpack_params(torch.as_tensor(phys, dtype=_FDTYPE), *self.ref)
        return D.table_from_tensors(a, b, r, h, *self.Q, self.dev)

    def chi_grad(self, phys: np.ndarray):
        out, _ = D.misfit_gradient(self.table(phys), self.p, self.omega, self.R_obs, self.fs)
        out = out.cpu().numpy()
        return float(out[4 * self.L]), out[self.idx]

    def chi(self, phys: np.ndarray) -> float:
        R = D.reflectivity(self.table(phys), self.p, self.omega, self.fs)
        r = R - self.R_obs
        return float((r.real**2 + r.imag**2).sum())

    def _models(self, rows: np.ndarray) -> list:
        out = []
        for m in rows:
            a, b, r, h = _unpack_params(torch.as_tensor(m, dtype=_FDTYPE), *self.ref)
            out.append(LayerModel(a.numpy(), b.numpy(), r.numpy(), h.numpy(), self.Q[0].numpy(),
                                  self.Q[1].numpy()))
        return out

    # central-difference stencils of the gradient: (offsets in steps, weights); column j of H
    # is sum_k w_k g(m + o_k d_j e_j) / d_j
    _STENCILS = {2: ((1, -1), (0.5, -0.5)),
                 4: ((2, 1, -1, -2), (-1.0 / 12, 8.0 / 12, -8.0 / 12, 1.0 / 12))}

    def basis(self) -> torch.Tensor:
        """Unit directions of the packed parameters in the full [4L] parameter space."""
        P = len(self.idx)
        V = torch.zeros((P, 4 * self.L), dtype=_FDTYPE, device=self.dev)
        V[torch.arange(P), torch.as_tensor(self.idx)] = 1.0
        return V

    def hessian_exact(self, phys: np.ndarray) -> np.ndarray:
        """The exact Hessian over the packed parameters: H e_j for every j from one launch of
        the tangent-of-adjoint kernel (kr_misfit_hvp), symmetrised."""
        HV = D.misfit_hvp(self.table(phys), self.p, self.omega, self.R_obs, self.basis(), self.fs)
        H = HV[:, self.idx].cpu().numpy()
        return 0.5 * (H + H.T)

    def hessian_fd(self, phys: np.ndarray, step: float = 1e-5, stencil: int = 2) -> np.ndarray:
        """Central differences of the exact adjoint gradient, all perturbed models in one
        batched launch (the batch is built on the first call and updated in place after).
        ``stencil`` 2 (error O(d^2): ~1e-7 relative at the default step) or 4 (fourth order,
        four gradients per parameter: ~1e-10 relative).  A cross-check of hessian_exact."""
        from .batch import BatchItem, ModelBatch

        rows, d = self.stencil_rows(phys, step, stencil)
        P, K = len(phys), len(self._STENCILS[stencil][0])
        models = self._models(rows)
        batch = getattr(self, "_hbatch", None)
        if batch is None or len(batch.desc) != K * P:
            items = [BatchItem(m, self.p, self.omega, gradient=True, R_obs=self.R_obs,
                               free_surface=self.fs) for m in models]
            batch = self._hbatch = ModelBatch(items, device=self.dev)
        else:
            batch.update_layers(models)
        batch.launch()
        # every item is a gradient model with L layers: rows of 4L + 1 (gradient, chi) in order
        rows = batch.chi_grad[:K * P * (4 * self.L + 1)].view(K * P, 4 * self.L + 1)
        return self.stencil_hessian(rows[:, self.idx].cpu().numpy(), d, stencil)

    @classmethod
    def stencil_rows(cls, phys: np.ndarray, step: float, stencil: int):
        """The K * P perturbed parameter rows of a stencil (block k: every parameter moved by
        offset k times its step) and the steps d."""
        offs = cls._STENCILS[stencil][0]
        P = len(phys)
        d = step * np.maximum(np.abs(phys), 1e-3)
        rows = np.repeat(np.asarray(phys, dtype=np.float64)[None, :], len(offs) * P, axis=0)
        for k, o in enumerate(offs):
            rows[k * P + np.arange(P), np.arange(P)] += o * d
        return rows, d

    @classmethod
    def stencil_hessian(cls, g: np.ndarray, d: np.ndarray, stencil: int) -> np.ndarray:
        """Symmetrised Hessian from the gradients g (K * P rows, in stencil_rows order)."""
        wts = cls._STENCILS[stencil][1]
        P = len(d)
        H = sum(w * g[k * P:(k + 1) * P] for k, w in enumerate(wts)).T / d[None, :]
        return 0.5 * (H + H.T)

    def hessian_gn(self, phys: np.ndarray) -> np.ndarray:
        _, J = D.jacobian(self.table(phys), self.p, self.omega, self.fs, want_R=False)
        Jp = J[:, self.idx, :]  # (n_p, P, n_w)
        H = 2.0 * torch.einsum("jaw,jbw->ab", Jp.conj(), Jp).real
        return H.cpu().numpy()


def taup_misfit_grad_hessian(log_params, alpha_ref, beta_ref, rho_ref, thickness_ref, Q_alpha,
                             Q_beta, p_values, omega, R_obs, hessian: str = "exact"):
    """``(chi, g_log, H_log)`` summed over all slownesses (``taup_inversion.py:112-187``)."""
    prob = _Problem(alpha_ref, beta_ref, rho_ref, thickness_ref, Q_alpha, Q_beta, p_values,
                    omega, R_obs)
    return _chi_g_h(prob, np.asarray(log_params, dtype=np.float64), hessian)


def _chi_g_h(prob: _Problem, log_params: np.ndarray, hessian: str):
    m = np.exp(log_params)
    chi, g = prob.chi_grad(m)
    if hessian == "exact":
        H = prob.hessian_exact(m)
    elif hessian in ("gauss-newton", "gn"):
        H = prob.hessian_gn(m)
    else:
        raise ValueError(f"hessian must be 'exact' or 'gauss-newton', got {hessian!r}")
    g_log = m * g
    H_log = np.outer(m, m) * H + np.diag(g * m)
    return chi, g_log, H_log


def newton_lm_step(g: np.ndarray, H: np.ndarray, lam: float) -> np.ndarray:
    """Solve (H + lambda I) dx = -g (``taup_inversion.py:238-254``)."""
    return np.linalg.solve(H + lam * np.eye(len(g)), -g)


def _to_layer_model(a, b, r, h, ref: LayerModel) -> LayerModel:
    h = np.asarray(h, dtype=np.float64).copy()
    h[h >= 1e29] = np.inf
    return LayerModel.from_arrays(np.asarray(a), np.asarray(b), np.asarray(r), h, ref.Q_alpha,
                                  ref.Q_beta)


def invert_taup(true_model: LayerModel, p_values, nfreq: int = 64, perturbation: float = 0.15,
                max_iter: int = 100, seed: int = 42, tol: float = 1e-8,
                hessian: str = "exact", initial_params: np.ndarray | None = None) -> InversionResult:
    """Newton-LM tau-p inversion (``taup_inversion.py:262-470``), GPU-backed.

    Same data generation (omega_k = k 2pi/64, k = 1..nfreq), same uniform initial perturbation
    scheme and seed semantics, same damping rules and convergence tests.  ``initial_params``
    (packed physical parameters) overrides the perturbation draw.
    """
    t = model_to_tensors(true_model)
    T = 64.0
    dw = 2.0 * np.pi / T
    omega = torch.arange(1, nfreq + 1, dtype=_FDTYPE) * dw
    dev = D.require_cuda()
    tab_true = D.table_from_tensors(t["alpha"], t["beta"], t["rho"], t["thickness"],
                                    t["Q_alpha"], t["Q_beta"], dev)
    p_arr = np.asarray(p_values, dtype=np.float64)
    R_obs = D.reflectivity(tab_true, p_arr, omega)
    true_params = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"]).numpy()
    n_params = len(true_params)
    n_sub = true_model.n_layers - 1
    if initial_params is None:
        rng = np.random.default_rng(seed)
        perturb = np.ones(n_params)
        n_vel = 2 * n_sub
        perturb[:n_vel] = rng.uniform(1.0 - perturbation, 1.0 + perturbation, n_vel)
        perturb[n_vel:n_vel + n_sub] = rng.uniform(1.0 - perturbation * 0.67,
                                                   1.0 + perturbation * 0.67, n_sub)
        perturb[n_vel + n_sub:] = rng.uniform(1.0 - perturbation * 1.33,
                                              1.0 + perturbation * 1.33, n_sub - 1)
        init_params = true_params * perturb
    else:
        init_params = np.asarray(initial_params, dtype=np.float64)
    prob = _Problem(t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"],
                    p_arr, omega, R_obs)
    a_i, b_i, r_i, h_i = _unpack_params(torch.as_tensor(init_params), *prob.ref)
    initial_model = _to_layer_model(a_i, b_i, r_i, h_i, true_model)
    log_x = np.log(init_params)
    misfit_history, grad_norm_history, param_error_history = [], [], []
    lam = None
    for iteration in range(max_iter):
        chi, g, H = _chi_g_h(prob, log_x, hessian)
        grad_norm = float(np.linalg.norm(g))
        param_err = float(np.linalg.norm(np.exp(log_x) - true_params) / np.linalg.norm(true_params))
        misfit_history.append(chi)
        grad_norm_history.append(grad_norm)
        param_error_history.append(param_err)
        logger.info("iter %3d  chi=%.4e  ||g||=%.4e  err=%.4e", iteration, chi, grad_norm,
                    param_err)
        if lam is None:
            lam = 0.01 * max(float(np.abs(np.diag(H)).max()), 1e-10)
        if grad_norm < tol:
            break
        if len(misfit_history) > 1:
            rel_change = abs(misfit_history[-2] - chi) / max(abs(chi), 1e-30)
            if rel_change < tol:
                break
        accepted = False
        for _ in range(10):
            dx = newton_lm_step(g, H, lam)
            trial_x = log_x + dx
            if prob.chi(np.exp(trial_x)) < chi:
                log_x = trial_x
                lam = max(lam / 2.0, 1e-15)
                accepted = True
                break
            lam *= 5.0
        if not accepted:
            logger.warning("Line search failed at iteration %d", iteration)
            break
    a_r, b_r, r_r, h_r = _unpack_params(torch.as_tensor(np.exp(log_x)), *prob.ref)
    recovered = _to_layer_model(a_r, b_r, r_r, h_r, true_model)
    converged = bool(param_error_history and param_error_history[-1] < 0.01)
    return InversionResult(true_model=true_model, initial_model=initial_model,
                           recovered_model=recovered, misfit_history=misfit_history,
                           grad_norm_history=grad_norm_history,
                           param_error_history=param_error_history,
                           n_iterations=len(misfit_history), converged=converged)


def compute_taup_traces(model: LayerModel, p_values, T: float = 64.0, nw: int = 1024):
    """Ricker-convolved tau-p traces (``taup_inversion.py:527-571``): one launch for all p."""
    dev = D.require_cuda()
    dw = 2.0 * np.pi / T
    omega = np.arange(1, nw, dtype=np.float64) * dw
    S = ricker_spectrum(omega, nw * dw)
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    R = D.reflectivity(D.layer_table(model, dev), np.asarray(p_values, dtype=np.float64), omega)
    tr = D.traces(R, nw, S=S).cpu().numpy()
    return time, {p: tr[i] for i, p in enumerate(p_values)}
