"""Drop-in for ``Kennett_Reflectivity.kennett_torch`` (``kennett_torch.py:312-725``).

``kennett_reflectivity_torch`` keeps the reference signature and returns the same complex128
R(omega), differentiable with respect to ``alpha, beta, rho, thickness``, through a
``torch.autograd.Function`` over the hand-written adjoint kernels:

* plain inference computes R only (``kr_reflectivity``);
* ``backward()`` / ``torch.autograd.grad`` run the vector-Jacobian product kernel
  (``kr_vjp``) with the upstream gradient: one reverse sweep per (p, omega) that recomputes
  the forward layer by layer, so no Jacobian and no per-layer intermediates are stored,
  whatever n_omega * n_p * layers;
* ``torch.func`` transforms (``jacrev`` / ``jacfwd`` / ``vjp`` / ``jvp`` / ``vmap``) and
  forward-mode AD get R and the Jacobian (``kr_jacobian``) and contract it with tensor
  operations.  The Jacobian is itself differentiable: its tangent is the second derivative
  of R along the input tangent (``kr_jacobian_dot``, the tangent of the adjoint), so
  ``torch.func.hessian`` of a misfit built on the Function -- forward over reverse, as the
  reference's ``hessian`` and ``invert_taup`` take it -- is the exact Hessian, and reverse
  over reverse contracts the full second-derivative tensor.  ``hessian()`` below gives the
  exact Hessian of the misfit in one launch.

``Q_alpha``, ``Q_beta``, ``p`` and ``omega`` are constants (no gradient).

Inputs may live on the CPU (as in the reference) or on a CUDA device; the result is returned
on ``omega``'s device.
"""

from __future__ import annotations

import numpy as np
import torch

from . import device as D
from .layer_model import LayerModel

__all__ = [
    "kennett_reflectivity_torch",
    "forward_model_torch",
    "jacobian",
    "hessian",
    "model_to_tensors",
    "misfit_gradient_packed",
]

_CDTYPE = torch.complex128
_FDTYPE = torch.float64


def _device_for(*tensors) -> torch.device:
    for t in tensors:
        if isinstance(t, torch.Tensor) and t.is_cuda:
            return D.require_cuda(t.device)
    return D.require_cuda()


# How much derivative information a forward call must produce:
#   NONE : R only (no input needs a derivative);
#   VJP  : R only; backward() runs the adjoint kernel kr_vjp with the upstream gradient
#          (plain torch.autograd: the Jacobian is never formed, the adjoint recomputes the
#          forward per layer);
#   JAC  : R and the Jacobian J [n_p, 4L, n_w] (functorch transforms -- jacrev, jacfwd,
#          vmap, hessian -- and forward-mode AD contract J with tensor operations).
_NONE, _VJP, _JAC = 0, 1, 2


def _compute(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, need_jac):
    """R (and J if ``need_jac``) for the given layer arrays, on the compute device.

    Returns ``(R [n_p, n_w], J [n_p, 4L, n_w] or None)``.
    """
    dev = _device_for(alpha, omega)
    tab = D.table_from_tensors(alpha, beta, rho, thickness, Q_alpha, Q_beta, dev)
    p_t = torch.as_tensor(p, dtype=_FDTYPE).detach().reshape(-1)
    w = torch.as_tensor(omega).detach()
    if need_jac:
        return D.jacobian(tab, p_t, w, free_surface)
    return D.reflectivity(tab, p_t, w, free_surface), None


def _jacobian_dot(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, V):
    """d/dv of the Jacobian for directions V [n_dir, 4L]: [n_dir, n_p, 4L, n_w] complex on the
    compute device (``kr_jacobian_dot``, the tangent of the adjoint)."""
    dev = _device_for(alpha, omega)
    tab = D.table_from_tensors(alpha, beta, rho, thickness, Q_alpha, Q_beta, dev)
    p_t = torch.as_tensor(p, dtype=_FDTYPE).detach().reshape(-1)
    return D.jacobian_dot(tab, p_t, torch.as_tensor(omega).detach(), V, free_surface)


def _second_derivatives(args, free_surface, L):
    """d^2 R / d theta_m d theta_k for every m: [4L, n_p, 4L, n_w] (one launch over the basis)."""
    with torch._C._DisableFuncTorch():
        V = torch.eye(4 * L, dtype=_FDTYPE)
        return _jacobian_dot(*args, free_surface, V)


def _vjp(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, gR):
    """grad [4L] = Re sum_{p, w} conj(gR) dR/dtheta by the adjoint kernel (``kr_vjp``)."""
    dev = _device_for(alpha, omega)
    tab = D.table_from_tensors(alpha, beta, rho, thickness, Q_alpha, Q_beta, dev)
    p_t = torch.as_tensor(p, dtype=_FDTYPE).detach().reshape(-1)
    g, _ = D.vjp(tab, p_t, torch.as_tensor(omega).detach(), gR, free_surface)
    return g


def _value(t, dtype=None) -> torch.Tensor:
    """The plain value of a tensor that torch.func transforms may have wrapped (grad / jvp
    levels), optionally converted: the kernels read raw device memory."""
    t = torch.as_tensor(t)
    while torch._C._functorch.is_functorch_wrapped_tensor(t):
        t = torch._C._functorch.get_unwrapped(t)
    with torch._C._DisableFuncTorch():
        t = t.detach()
        return t if dtype is None else t.to(dtype)


def _plain_call(fn, *args):
    """Runs a kernel wrapper outside the active torch.func transforms, so that the tensors it
    creates are plain device memory (its result enters the transformed computation as a
    constant)."""
    with torch._C._DisableFuncTorch():
        return fn(*args)


def _split(g, L, ctx):
    """Per-parameter slices of a [..., 4L] gradient on the inputs' devices and dtypes."""
    return tuple(g[..., k * L:(k + 1) * L].to(device=ctx.devices[k], dtype=ctx.dtypes[k])
                 for k in range(4)) + (None,) * 6


class _KennettFunction(torch.autograd.Function):
    """R(alpha, beta, rho, thickness) with the hand-written adjoint as its derivative.

    Outputs ``(R, J)``; J is the Jacobian in JAC mode and an empty placeholder otherwise.
    """

    @staticmethod
    def forward(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, mode):
        R, J = _compute(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface,
                        mode == _JAC)
        out_dev = omega.device
        scalar_p = torch.as_tensor(p).dim() == 0
        R = R.to(out_dev)
        if J is None:
            J = torch.empty(0, dtype=_CDTYPE, device=out_dev)
        else:
            J = J.to(out_dev)
            if scalar_p:
                J = J[0]
        if scalar_p:
            R = R[0]
        return R, J

    @staticmethod
    def setup_context(ctx, inputs, output):
        _, J = output
        ctx.mode = inputs[9]
        ctx.L = inputs[0].shape[0]
        ctx.dtypes = [x.dtype for x in inputs[:4]]
        ctx.devices = [x.device for x in inputs[:4]]
        ctx.free_surface = inputs[8]
        ctx.scalar_p = torch.as_tensor(inputs[6]).dim() == 0
        # the layer inputs themselves (a differentiable backward re-enters through them) and
        # the constants as float64 (a Python float p would otherwise become float32)
        layer = [torch.as_tensor(x) for x in inputs[:4]]
        const = [torch.as_tensor(x, dtype=_FDTYPE).detach() for x in inputs[4:7]]
        const.append(torch.as_tensor(inputs[7]).detach())
        if ctx.mode == _JAC:
            # J is differentiable: its tangent (jvp) is the second derivative along the input
            # tangent, so forward over reverse (torch.func.hessian) is exact
            ctx.save_for_backward(J, *layer, *const)
            ctx.save_for_forward(J, *layer, *const)
        else:
            ctx.mark_non_differentiable(J)
            ctx.save_for_backward(*layer, *const)

    @staticmethod
    def _model(saved):
        """Value-only model arguments (alpha .. omega) from the saved tensors."""
        return [_value(x, _FDTYPE) for x in saved[:4]] + [_value(x) for x in saved[4:8]]

    @staticmethod
    def backward(ctx, gR, gJ):
        L = ctx.L
        if ctx.mode == _JAC:
            J, *saved = ctx.saved_tensors
            args = _KennettFunction._model(saved)
        else:
            saved = ctx.saved_tensors
            args = _KennettFunction._model(saved)
            wrapped = torch._C._functorch.is_functorch_wrapped_tensor(gR)
            if not wrapped and not torch.is_grad_enabled():
                # the adjoint kernel: one reverse sweep per (p, omega), no Jacobian formed
                return _split(_plain_call(_vjp, *args, ctx.free_surface, _value(gR)), L, ctx)
            if torch.is_grad_enabled() and not wrapped:
                # a differentiable backward (create_graph=True): the Jacobian as a
                # differentiable function of the layer inputs (JAC mode), so that a second
                # backward sees second derivatives
                _, J = _KennettFunction.apply(*saved[:8], ctx.free_surface, _JAC)
            else:
                # a transformed backward (vmap over cotangents): contract the Jacobian with
                # tensor operations
                _, J = _plain_call(_compute, *args, ctx.free_surface, True)
                if ctx.scalar_p:
                    J = J[0]
            J = J.to(gR.device)
        # d loss / d theta = Re(sum_w conj(gR[w]) J[theta, w])  (PyTorch complex convention)
        g = (gR.conj().unsqueeze(-2) * J).real.sum(-1)
        if g.dim() > 1:
            g = g.sum(-2)
        if ctx.mode == _JAC and gJ is not None:
            # reverse over reverse: sum conj(gJ) d^2 R / d theta_m d theta_k over k, p, omega
            T = _second_derivatives(args, ctx.free_surface, L).to(gJ.device)
            if ctx.scalar_p:
                T = T[:, 0]
            g2 = (gJ.conj().unsqueeze(0) * T).real
            g = g + g2.reshape(4 * L, -1).sum(-1)
        return _split(g, L, ctx)

    @staticmethod
    def vmap(info, in_dims, alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
             free_surface, mode):
        # One evaluation per batch element (each is one kernel launch over all p and omega).
        args = (alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega)
        Rs, Js = [], []
        for b in range(info.batch_size):
            sl = [x if d is None else x.select(d, b) for x, d in zip(args, in_dims[:8])]
            R, J = _KennettFunction.apply(*sl, free_surface, mode)
            Rs.append(R)
            Js.append(J)
        return (torch.stack(Rs), torch.stack(Js)), (0, 0)

    @staticmethod
    def jvp(ctx, ta, tb, tr, th, tqa, tqb, tp, tw, tfs, tmode):
        J, *saved = ctx.saved_tensors
        args = _KennettFunction._model(saved)
        L = ctx.L
        parts = []
        for t in (ta, tb, tr, th):
            parts.append(torch.zeros(L, dtype=_FDTYPE, device=J.device) if t is None
                         else t.to(device=J.device, dtype=_FDTYPE))
        v = torch.cat(parts)
        dR = (J * v.to(_CDTYPE).unsqueeze(-1)).sum(-2)
        if torch._C._functorch.is_functorch_wrapped_tensor(v):
            # a batch of tangents (jacfwd, hessian): contract the second-derivative tensor with
            # tensor operations, which the transform batches
            T = _second_derivatives(args, ctx.free_surface, L).to(J.device)
            if ctx.scalar_p:
                T = T[:, 0]
            dJ = (T * v.to(_CDTYPE).reshape((4 * L,) + (1,) * (T.dim() - 1))).sum(0)
        else:
            with torch._C._DisableFuncTorch():
                dJ = _jacobian_dot(*args, ctx.free_surface, _value(v).reshape(1, -1))[0]
            dJ = dJ.to(J.device)
            if ctx.scalar_p:
                dJ = dJ[0]
        return dR, dJ


def _derivative_mode(*tensors) -> int:
    """JAC when a functorch transform or forward-mode AD sees the layer inputs, VJP when only
    plain reverse-mode autograd needs their gradient, else NONE."""
    mode = _NONE
    for t in tensors:
        if not isinstance(t, torch.Tensor):
            continue
        if torch._C._functorch.is_functorch_wrapped_tensor(t):
            return _JAC
        try:
            if torch.autograd.forward_ad.unpack_dual(t).tangent is not None:
                return _JAC
        except RuntimeError:
            pass
        if t.requires_grad and torch.is_grad_enabled():
            mode = _VJP
    return mode


def _needs_grad(*tensors) -> bool:
    """Whether any layer input carries reverse- or forward-mode derivative information."""
    return _derivative_mode(*tensors) != _NONE


def kennett_reflectivity_torch(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                               free_surface: bool = False):
    """Complex PP reflectivity (nfreq,) -- ``kennett_torch.py:312-480`` signature.

    ``p`` may also be a 1-D tensor of slownesses, giving R of shape (n_p, nfreq) in one
    launch.  The half-space may be marked by a thickness >= 1e30 (the reference's sentinel) or
    +inf.
    """
    if not isinstance(omega, torch.Tensor):
        omega = torch.as_tensor(omega)
    mode = _derivative_mode(alpha, beta, rho, thickness)
    R, _ = _KennettFunction.apply(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                                  bool(free_surface), mode)
    return R


def forward_model_torch(alpha, beta, rho, thickness, Q_alpha, Q_beta, p: float, T: float = 64.0,
                        nw: int = 2048, free_surface: bool = False):
    """``(time, seismogram)`` (``kennett_torch.py:488-544``): R x Ricker, Hermitian FFT.

    R is differentiable (adjoint kernel); the spectrum assembly and FFT are torch ops on the
    result's device.
    """
    dw = 2.0 * np.pi / T
    nwm = nw - 1
    wmax = nw * dw
    dev = alpha.device if isinstance(alpha, torch.Tensor) else torch.device("cpu")
    omega = torch.arange(1, nwm + 1, dtype=_FDTYPE, device=dev) * dw
    a = 0.1 * wmax
    t0 = 5.0 / (a * (2.0**0.5))
    Z = (omega**2) / (4.0 * a**2)
    S = Z * torch.exp(-Z + 1j * omega * t0)
    R = kennett_reflectivity_torch(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                                   free_surface=free_surface)
    Y = R * S
    nt = 2 * nw
    Uwk = torch.cat([torch.zeros(1, dtype=_CDTYPE, device=dev), Y,
                     torch.zeros(1, dtype=_CDTYPE, device=dev), torch.conj(torch.flip(Y, [0]))])
    time = torch.arange(nt, dtype=_FDTYPE, device=dev) * (T / float(nt))
    return time, torch.fft.fft(Uwk).real


# ---------------------------------------------------------------------------------------
# Packed sub-ocean parameters (kennett_torch.py:552-608)
# ---------------------------------------------------------------------------------------

def _pack_params(alpha, beta, rho, thickness):
    """m = [Vp_1..N, Vs_1..N, rho_1..N, h_1..N-1] (ocean and half-space thickness excluded)."""
    return torch.cat([alpha[1:], beta[1:], rho[1:], thickness[1:-1]])


def _unpack_params(params, alpha_full, beta_full, rho_full, thickness_full):
    n_sub = alpha_full.shape[0] - 1
    n_thick = n_sub - 1
    a = params[:n_sub]
    b = params[n_sub:2 * n_sub]
    r = params[2 * n_sub:3 * n_sub]
    h = params[3 * n_sub:3 * n_sub + n_thick]
    return (torch.cat([alpha_full[:1].detach(), a]), torch.cat([beta_full[:1].detach(), b]),
            torch.cat([rho_full[:1].detach(), r]),
            torch.cat([thickness_full[:1].detach(), h, thickness_full[-1:].detach()]))


def packed_index(L: int) -> list[int]:
    """Rows of the full [4L] layer-parameter vector that form the packed vector."""
    return ([0 * L + l for l in range(1, L)] + [1 * L + l for l in range(1, L)]
            + [2 * L + l for l in range(1, L)] + [3 * L + l for l in range(1, L - 1)])


def jacobian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p: float, omega,
             free_surface: bool = False) -> torch.Tensor:
    """dR(omega_i)/dm_j, shape (nfreq, 4N-1) complex (``kennett_torch.py:611-641``).

    One launch of the adjoint kernel (the reference runs jacrev twice, for Re and Im).
    Returned on ``omega``'s device.
    """
    omega = torch.as_tensor(omega)
    _, J = _compute(alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega, free_surface, True)
    L = torch.as_tensor(alpha).shape[0]
    Jp = J[0][packed_index(L)].transpose(0, 1).contiguous()
    return Jp.to(omega.device)


def misfit_gradient_packed(params, alpha, beta, rho, thickness, Q_alpha, Q_beta, p, omega,
                           R_obs, free_surface: bool = False):
    """(chi, d chi / d m) for packed parameters m, all slownesses ``p`` in one launch.

    chi = sum_{p, w} |R - R_obs|^2; ``R_obs`` has shape (n_p, n_w) (or (n_w,) for one p).
    Returns ``(chi float, grad float64 tensor on the compute device)``.
    """
    a, b, r, h = _unpack_params(torch.as_tensor(params, dtype=_FDTYPE).detach().cpu(),
                                *(torch.as_tensor(x, dtype=_FDTYPE).cpu() for x in
                                  (alpha, beta, rho, thickness)))
    dev = _device_for(omega, R_obs)
    tab = D.table_from_tensors(a, b, r, h, Q_alpha, Q_beta, dev)
    p_t = torch.as_tensor(p, dtype=_FDTYPE).reshape(-1)
    Ro = torch.as_tensor(R_obs).reshape(p_t.numel(), -1)
    out, _ = D.misfit_gradient(tab, p_t, torch.as_tensor(omega), Ro, free_surface)
    L = a.shape[0]
    return float(out[4 * L]), out[packed_index(L)]


def hessian(alpha, beta, rho, thickness, Q_alpha, Q_beta, p: float, omega, R_obs=None,
            free_surface: bool = False) -> torch.Tensor:
    """Hessian of chi = ||R - R_obs||^2 over the packed parameters (``kennett_torch.py:644-684``).

    Exact: column j is H e_j from the tangent-of-adjoint kernel (``kr_misfit_hvp``, all
    columns in one launch; forward-mode dual numbers through the adjoint, no step size), the
    second derivative the reference's torch.func.hessian takes by reverse over reverse.
    Returned on ``omega``'s device as float64 (n_params, n_params), symmetrised.
    """
    from .taup_inversion import _Problem

    omega = torch.as_tensor(omega)
    if R_obs is None:
        R_obs = torch.zeros(omega.shape[0], dtype=_CDTYPE)
    m0 = _pack_params(*(torch.as_tensor(x, dtype=_FDTYPE).detach().cpu()
                        for x in (alpha, beta, rho, thickness)))
    prob = _Problem(alpha, beta, rho, thickness, Q_alpha, Q_beta, [float(p)], omega,
                    torch.as_tensor(R_obs).reshape(1, -1), free_surface=free_surface)
    H = prob.hessian_exact(m0.numpy())
    return torch.as_tensor(H, dtype=_FDTYPE).to(omega.device)


def model_to_tensors(model: LayerModel, requires_grad: bool = False) -> dict:
    """Dict of float64 tensors; half-space thickness -> 1e30 (``kennett_torch.py:692-725``)."""
    thick = model.thickness.copy()
    thick[np.isinf(thick)] = 1e30
    out = {}
    for name, arr in [("alpha", model.alpha), ("beta", model.beta), ("rho", model.rho),
                      ("thickness", thick), ("Q_alpha", model.Q_alpha), ("Q_beta", model.Q_beta)]:
        t = torch.tensor(arr, dtype=_FDTYPE)
        if requires_grad and name in ("alpha", "beta", "rho", "thickness"):
            t.requires_grad_(True)
        out[name] = t
    return out
