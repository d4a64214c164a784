"""Many tau-p Newton-LM inversions at once, with the LM state on the device.

``invert_taup_batch`` runs K independent inversions of ``invert_taup``
(``Kennett_Reflectivity/taup_inversion.py:262-470``: log-parameter Newton-LM, lambda0 =
0.01 max|diag H|, accept -> lambda / 2 (floor 1e-15), reject -> lambda * 5, at most 10 trials,
stop on ||g|| < tol or relative misfit change < tol) in lockstep.  Per iteration:

* the misfit gradients of all K current points are one batched adjoint launch
  (``kr_batch_launch``); the exact Hessian (``hessian="exact"``) is one tangent-of-adjoint
  launch per inversion (``kr_misfit_hvp``, every packed direction at once), the Gauss-Newton
  Hessian 2 Re(J^H J) one ``kr_jacobian`` launch per inversion;
* the log transform, the damping initialisation, the K damped (H + lambda I) solves
  (batched ``torch.linalg.solve``), the trial points and their layer tables are device
  tensor operations;
* the K trial misfits are one batched forward launch; acceptance, the lambda updates and the
  convergence tests are masks on the device.

The host reads one flag per trial round (whether any inversion still searches) and one per
iteration (whether any is still running): the round trips of K inversions are shared instead
of paid K times.  All inversions must have the same layer count and share p and omega.
"""

from __future__ import annotations

import numpy as np
import torch

from . import device as D
from .batch import BatchItem, ModelBatch
from .kennett_torch import _pack_params, _unpack_params, model_to_tensors, packed_index
from .layer_model import LayerModel
from .taup_inversion import InversionResult, _to_layer_model

__all__ = ["invert_taup_batch"]

_F = torch.float64
_C = torch.complex128


def _draw_start(true_params: np.ndarray, n_sub: int, perturbation: float, seed: int):
    """The reference's uniform perturbation of the true parameters (``taup_inversion.py:330-347``)."""
    rng = np.random.default_rng(seed)
    perturb = np.ones(len(true_params))
    n_vel = 2 * n_sub
    perturb[:n_vel] = rng.uniform(1.0 - perturbation, 1.0 + perturbation, n_vel)
    perturb[n_vel:n_vel + n_sub] = rng.uniform(1.0 - perturbation * 0.67,
                                               1.0 + perturbation * 0.67, n_sub)
    perturb[n_vel + n_sub:] = rng.uniform(1.0 - perturbation * 1.33,
                                          1.0 + perturbation * 1.33, n_sub - 1)
    return true_params * perturb


class _Tables:
    """Layer tables [M, 6, L] on the device from packed physical parameters [M, P]."""

    def __init__(self, ref: torch.Tensor):
        self.ref = ref  # [K, 6, L]: ocean values, half-space thickness and Q from the models
        self.L = ref.shape[2]
        self.n_sub = self.L - 1

    def __call__(self, x: torch.Tensor, owner: torch.Tensor) -> torch.Tensor:
        n, L = self.n_sub, self.L
        ref = self.ref[owner]
        tab = ref.clone()
        tab[:, 0, 1:] = x[:, :n]
        tab[:, 1, 1:] = x[:, n:2 * n]
        tab[:, 2, 1:] = x[:, 2 * n:3 * n]
        tab[:, 3, 1:L - 1] = x[:, 3 * n:]
        return tab


def invert_taup_batch(true_models: list[LayerModel], p_values, nfreq: int = 64,
                      perturbation: float = 0.15, max_iter: int = 100,
                      seeds: list[int] | None = None, tol: float = 1e-8,
                      hessian: str = "gauss-newton", initial_params=None) -> list[InversionResult]:
    """K concurrent Newton-LM tau-p inversions; returns one ``InversionResult`` each.

    ``seeds`` (default 42 for every inversion) and ``initial_params`` (list of packed physical
    parameter vectors) have the meaning of ``invert_taup``'s ``seed`` / ``initial_params``.
    """
    if hessian not in ("gauss-newton", "gn", "exact"):
        raise ValueError(f"hessian must be 'exact' or 'gauss-newton', got {hessian!r}")
    K = len(true_models)
    if K == 0:
        return []
    L = true_models[0].n_layers
    if any(m.n_layers != L for m in true_models):
        raise ValueError("all inversions of a batch need the same layer count")
    dev = D.require_cuda()
    seeds = list(seeds) if seeds is not None else [42] * K
    dw = 2.0 * np.pi / 64.0
    omega = torch.arange(1, nfreq + 1, dtype=_F, device=dev) * dw
    w_c = omega.to(_C)
    p_arr = np.asarray(p_values, dtype=np.float64)
    p_t = torch.as_tensor(p_arr, device=dev)
    n_p, n_w = len(p_arr), nfreq
    idx = torch.as_tensor(packed_index(L), device=dev)

    tabs_true, true_params, starts = [], [], []
    for k, m in enumerate(true_models):
        t = model_to_tensors(m)
        tp = _pack_params(t["alpha"], t["beta"], t["rho"], t["thickness"]).numpy()
        true_params.append(tp)
        tabs_true.append(D.layer_table(m, dev))
        if initial_params is not None:
            starts.append(np.asarray(initial_params[k], dtype=np.float64))
        else:
            starts.append(_draw_start(tp, L - 1, perturbation, seeds[k]))
    ref = torch.stack(tabs_true)  # [K, 6, L]
    ref[:, 3, -1] = torch.where(torch.isinf(ref[:, 3, -1]), torch.full_like(ref[:, 3, -1], 1e30),
                                ref[:, 3, -1])
    tables = _Tables(ref)
    R_obs = torch.stack([D.reflectivity(tb, p_t, w_c) for tb in tabs_true])  # [K, n_p, n_w]
    P = len(true_params[0])
    x_true = torch.as_tensor(np.stack(true_params), device=dev)
    log_x = torch.log(torch.as_tensor(np.stack(starts), device=dev))

    # batches built once (shapes fixed); their layer buffers are rewritten on the device
    exact = hessian == "exact"
    per = 1
    owner_g = torch.arange(K, device=dev).repeat_interleave(per)
    obs = [R_obs[k] for k in range(K)]  # one object per inversion: its items share one copy
    items = [BatchItem(true_models[k], p_t, w_c, gradient=True, R_obs=obs[k])
             for k in range(K) for _ in range(per)]
    gbatch = ModelBatch(items, device=dev)
    fbatch = ModelBatch([BatchItem(true_models[k], p_t, w_c) for k in range(K)], device=dev)
    owner_f = torch.arange(K, device=dev)
    nv = 4 * L + 1

    basis = torch.zeros((P, 4 * L), dtype=_F, device=dev)
    basis[torch.arange(P), torch.as_tensor(idx)] = 1.0

    def grad_and_hessian(x_phys):
        gbatch.layers.view(-1, 6, L).copy_(tables(x_phys, owner_g))
        gbatch.launch()
        rows = gbatch.chi_grad[:len(items) * nv].view(K, per, nv)
        chi = rows[:, 0, 4 * L]
        g = rows[:, 0, :4 * L][:, idx]
        tabs = tables(x_phys, owner_f)
        H = torch.empty((K, P, P), dtype=_F, device=dev)
        for k in range(K):
            if exact:  # H e_j for every packed j: one tangent-of-adjoint launch
                HV = D.misfit_hvp(tabs[k].contiguous(), p_t, w_c, R_obs[k], basis)
                Hk = HV[:, idx]
                H[k] = 0.5 * (Hk + Hk.T)
            else:
                _, J = D.jacobian(tabs[k].contiguous(), p_t, w_c, want_R=False)
                Jp = J[:, idx, :]
                H[k] = 2.0 * torch.einsum("jaw,jbw->ab", Jp.conj(), Jp).real
        return chi, g, H

    def trial_misfit(x_phys):
        fbatch.layers.view(-1, 6, L).copy_(tables(x_phys, owner_f))
        fbatch.launch()
        R = fbatch.R[:K * n_p * n_w].view(K, n_p, n_w)
        r = R - R_obs
        return (r.real ** 2 + r.imag ** 2).sum(dim=(1, 2))

    active = torch.ones(K, dtype=torch.bool, device=dev)
    lam = torch.full((K,), float("nan"), dtype=_F, device=dev)
    prev_chi = torch.full((K,), float("nan"), dtype=_F, device=dev)
    hist_chi, hist_g, hist_err, hist_act = [], [], [], []
    eye = torch.eye(P, dtype=_F, device=dev)
    for _ in range(max_iter):
        m = torch.exp(log_x)
        chi, g_phys, H_phys = grad_and_hessian(m)
        g = m * g_phys
        H = m[:, :, None] * m[:, None, :] * H_phys + torch.diag_embed(g_phys * m)
        gnorm = torch.linalg.norm(g, dim=1)
        err = torch.linalg.norm(m - x_true, dim=1) / torch.linalg.norm(x_true, dim=1)
        hist_chi.append(chi.clone())
        hist_g.append(gnorm)
        hist_err.append(err)
        hist_act.append(active.clone())
        first = torch.isnan(lam)
        lam0 = 0.01 * torch.clamp(torch.diagonal(H, dim1=1, dim2=2).abs().amax(dim=1), min=1e-10)
        lam = torch.where(first, lam0, lam)
        rel = (prev_chi - chi).abs() / torch.clamp(chi.abs(), min=1e-30)
        conv = (gnorm < tol) | (~torch.isnan(prev_chi) & (rel < tol))
        searching = active & ~conv
        active = searching.clone()
        prev_chi = torch.where(active, chi, prev_chi)
        for _trial in range(10):
            if not bool(searching.any()):
                break
            # inversions that are not searching solve an identity system (dx = 0)
            Hs = torch.where(searching[:, None, None], H + lam[:, None, None] * eye, eye)
            gs = torch.where(searching[:, None], g, torch.zeros_like(g))
            dx = torch.linalg.solve(Hs, -gs)
            trial = log_x + dx
            chi_t = trial_misfit(torch.exp(trial))
            acc = searching & (chi_t < chi)
            log_x = torch.where(acc[:, None], trial, log_x)
            lam = torch.where(acc, torch.clamp(lam / 2.0, min=1e-15),
                              torch.where(searching, lam * 5.0, lam))
            searching = searching & ~acc
        active = active & ~searching  # line search failed: this inversion stops
        if not bool(active.any()):
            break

    chi_h = torch.stack(hist_chi).cpu().numpy()
    g_h = torch.stack(hist_g).cpu().numpy()
    e_h = torch.stack(hist_err).cpu().numpy()
    a_h = torch.stack(hist_act).cpu().numpy()
    x_fin = torch.exp(log_x).cpu().numpy()
    results = []
    for k, tm in enumerate(true_models):
        n_it = int(a_h[:, k].sum())
        t = model_to_tensors(tm)
        refs = [t["alpha"], t["beta"], t["rho"], t["thickness"]]
        init = _to_layer_model(*_unpack_params(torch.as_tensor(starts[k]), *refs), tm)
        rec = _to_layer_model(*_unpack_params(torch.as_tensor(x_fin[k]), *refs), tm)
        errs = list(map(float, e_h[:n_it, k]))
        results.append(InversionResult(
            true_model=tm, initial_model=init, recovered_model=rec,
            misfit_history=list(map(float, chi_h[:n_it, k])),
            grad_norm_history=list(map(float, g_h[:n_it, k])),
            param_error_history=errs, n_iterations=n_it,
            converged=bool(errs and errs[-1] < 0.01)))
    return results
