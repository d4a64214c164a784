"""Device-resident core: torch tensors in, torch tensors out, one C-ABI call per stage.

PyTorch supplies device memory (caching allocator), the current stream and host<->device
copies; every arithmetic step runs in ``libkennett_b200.so``.  Inputs and results stay on
the GPU, so callers that chain stages (reflectivity -> Bessel sum -> traces) never round-trip
through the host.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .layer_model import LayerModel, pack_layers

__all__ = [
    "require_cuda",
    "layer_table",
    "reflectivity",
    "bessel_sum",
    "traces",
    "jacobian",
    "misfit_gradient",
    "vjp",
    "misfit_hvp",
    "jacobian_dot",
    "table_from_tensors",
    "stream_handle",
]


def require_cuda(device=None) -> torch.device:
    """The CUDA device to run on; raises if none is visible (no CPU fallback)."""
    if not torch.cuda.is_available():
        raise RuntimeError("seismicinversion_b200 needs a CUDA GPU (sm_100a); none is visible")
    dev = torch.device("cuda") if device is None else torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"seismicinversion_b200 runs on CUDA devices only, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    _lib.lib()
    return dev


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def validate_table(tab: np.ndarray) -> None:
    tab = np.ascontiguousarray(tab, dtype=np.float64)
    _lib.check(_lib.lib().kr_validate_layers(tab.ctypes.data, tab.shape[1]), "layer model")


def layer_table(model: LayerModel, device=None) -> torch.Tensor:
    """Validated float64 ``[6, n_layers]`` layer table on the device."""
    dev = require_cuda(device)
    tab = pack_layers(model)
    validate_table(tab)
    return torch.from_numpy(tab).to(dev, non_blocking=False)


def _dev_f64(x, dev) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=dev)


def _dev_c128(x, dev) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.complex128).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.complex128), device=dev)


def reflectivity(layers: torch.Tensor, p, omega, free_surface: bool = False,
                 out: torch.Tensor | None = None) -> torch.Tensor:
    """R[p, omega] (complex128, device) for one model: ``kr_reflectivity``."""
    dev = layers.device
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    if out is None:
        out = torch.empty((n_p, n_w), dtype=torch.complex128, device=dev)
    elif out.shape != (n_p, n_w) or out.dtype != torch.complex128 or not out.is_contiguous():
        raise ValueError("out must be a contiguous complex128 tensor of shape (n_p, n_w)")
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    st = _lib.lib().kr_reflectivity(layers.data_ptr(), layers.shape[1], p_t.data_ptr(), n_p,
                                    w_t.data_ptr(), n_w, flags, out.data_ptr(),
                                    stream_handle(dev))
    _lib.check(st, "kr_reflectivity")
    return out


def gmm_reflectivity(layers: torch.Tensor, p, omega, free_surface: bool = False,
                     out: torch.Tensor | None = None) -> torch.Tensor:
    """R[p, omega] by the Global Matrix Method (block-Riccati sweep): ``kr_gmm_reflectivity``."""
    dev = layers.device
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    if out is None:
        out = torch.empty((n_p, n_w), dtype=torch.complex128, device=dev)
    elif out.shape != (n_p, n_w) or out.dtype != torch.complex128 or not out.is_contiguous():
        raise ValueError("out must be a contiguous complex128 tensor of shape (n_p, n_w)")
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    st = _lib.lib().kr_gmm_reflectivity(layers.data_ptr(), layers.shape[1], p_t.data_ptr(), n_p,
                                        w_t.data_ptr(), n_w, flags, out.data_ptr(),
                                        stream_handle(dev))
    _lib.check(st, "kr_gmm_reflectivity")
    return out


def bessel_sum(R: torch.Tensor, p, pw, dp: float, omega_real, offsets,
               out: torch.Tensor | None = None) -> torch.Tensor:
    """U[r, w] = sum_j R[j, w] ((pw_j w) dp) J0((w p_j) r): ``kr_bessel_sum``."""
    dev = R.device
    R = R.contiguous()
    p_t = _dev_f64(p, dev).reshape(-1)
    pw_t = _dev_f64(pw, dev).reshape(-1)
    w_t = _dev_f64(omega_real, dev).reshape(-1)
    r_t = _dev_f64(offsets, dev).reshape(-1)
    n_p, n_w, n_r = p_t.numel(), w_t.numel(), r_t.numel()
    if R.shape != (n_p, n_w) or R.dtype != torch.complex128:
        raise ValueError(f"R must be complex128 of shape ({n_p}, {n_w}), got {tuple(R.shape)}")
    h = _lib.lib()
    ws_bytes = h.kr_bessel_sum_workspace_bytes(n_p, n_w, n_r)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    if out is None:
        out = torch.empty((n_r, n_w), dtype=torch.complex128, device=dev)
    st = h.kr_bessel_sum(R.data_ptr(), p_t.data_ptr(), pw_t.data_ptr(), n_p, float(dp),
                         w_t.data_ptr(), n_w, r_t.data_ptr(), n_r, out.data_ptr(),
                         ws.data_ptr(), ws_bytes, stream_handle(dev))
    _lib.check(st, "kr_bessel_sum")
    return out


def traces(U: torch.Tensor, nw: int, S=None, decay=None,
           out: torch.Tensor | None = None) -> torch.Tensor:
    """Real traces (n_r, 2 nw) from spectra U (n_r, nw-1) times S: ``kr_traces``."""
    dev = U.device
    U = U.contiguous()
    if U.dim() == 1:
        U = U.reshape(1, -1)
    n_r = U.shape[0]
    if U.shape[1] != nw - 1 or U.dtype != torch.complex128:
        raise ValueError(f"U must be complex128 of shape (n_r, {nw - 1})")
    S_t = None if S is None else _dev_c128(S, dev).reshape(-1)
    d_t = None if decay is None else _dev_f64(decay, dev).reshape(-1)
    if S_t is not None and S_t.numel() != nw - 1:
        raise ValueError("S must have nw-1 values")
    if d_t is not None and d_t.numel() != 2 * nw:
        raise ValueError("decay must have 2*nw values")
    h = _lib.lib()
    ws_bytes = h.kr_traces_workspace_bytes(n_r, nw)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    if out is None:
        out = torch.empty((n_r, 2 * nw), dtype=torch.float64, device=dev)
    st = h.kr_traces(U.data_ptr(), _ptr(S_t), n_r, nw, _ptr(d_t), out.data_ptr(),
                     ws.data_ptr(), ws_bytes, stream_handle(dev))
    _lib.check(st, "kr_traces")
    return out


def jacobian(layers: torch.Tensor, p, omega, free_surface: bool = False,
             want_R: bool = True):
    """(R [n_p, n_w], J [n_p, 4L, n_w]) complex128 on the device: ``kr_jacobian``.

    J[j, k*L + l, w] = dR(p_j, w) / d theta with theta = alpha_l, beta_l, rho_l, h_l (k = 0..3).
    """
    dev = layers.device
    L = layers.shape[1]
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    h = _lib.lib()
    ws_bytes = h.kr_jacobian_workspace_bytes(L, n_p, n_w)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    R = torch.empty((n_p, n_w), dtype=torch.complex128, device=dev) if want_R else None
    J = torch.empty((n_p, 4 * L, n_w), dtype=torch.complex128, device=dev)
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    st = h.kr_jacobian(layers.data_ptr(), L, p_t.data_ptr(), n_p, w_t.data_ptr(), n_w, flags,
                       _ptr(R), J.data_ptr(), ws.data_ptr(), ws_bytes, stream_handle(dev))
    _lib.check(st, "kr_jacobian")
    return R, J


def misfit_gradient(layers: torch.Tensor, p, omega, R_obs, free_surface: bool = False,
                    want_R: bool = False):
    """chi = sum |R - R_obs|^2 and d chi / d theta [4L] on the device: ``kr_misfit_gradient``.

    Returns ``(chi_grad [4L + 1] float64 tensor (gradient then chi), R or None)``.
    """
    dev = layers.device
    L = layers.shape[1]
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    Ro = _dev_c128(R_obs, dev)
    if Ro.shape != (n_p, n_w):
        raise ValueError(f"R_obs must have shape ({n_p}, {n_w}), got {tuple(Ro.shape)}")
    h = _lib.lib()
    ws_bytes = h.kr_misfit_gradient_workspace_bytes(L, n_p, n_w)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    R = torch.empty((n_p, n_w), dtype=torch.complex128, device=dev) if want_R else None
    out = torch.empty(4 * L + 1, dtype=torch.float64, device=dev)
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    st = h.kr_misfit_gradient(layers.data_ptr(), L, p_t.data_ptr(), n_p, w_t.data_ptr(), n_w,
                              flags, Ro.data_ptr(), _ptr(R), out.data_ptr(), ws.data_ptr(),
                              ws_bytes, stream_handle(dev))
    _lib.check(st, "kr_misfit_gradient")
    return out, R


def vjp(layers: torch.Tensor, p, omega, gR, free_surface: bool = False, want_R: bool = False,
        out: torch.Tensor | None = None):
    """grad [4L] = Re sum_{p, w} conj(gR[p, w]) dR(p, w)/d theta on the device: ``kr_vjp``.

    ``gR`` is the cotangent of R (shape (n_p, n_w), complex); theta = (alpha, beta, rho, h) of
    every layer in the order of ``jacobian``.  Returns ``(grad, R or None)``.
    """
    dev = layers.device
    L = layers.shape[1]
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    g = _dev_c128(gR, dev)
    if g.numel() != n_p * n_w:
        raise ValueError(f"gR must have {n_p} x {n_w} values, got {tuple(g.shape)}")
    g = g.reshape(n_p, n_w).contiguous()
    h = _lib.lib()
    ws_bytes = h.kr_vjp_workspace_bytes(L, n_p, n_w)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    R = torch.empty((n_p, n_w), dtype=torch.complex128, device=dev) if want_R else None
    if out is None:
        out = torch.empty(4 * L, dtype=torch.float64, device=dev)
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    st = h.kr_vjp(layers.data_ptr(), L, p_t.data_ptr(), n_p, w_t.data_ptr(), n_w, flags,
                  g.data_ptr(), _ptr(R), out.data_ptr(), ws.data_ptr(), ws_bytes,
                  stream_handle(dev))
    _lib.check(st, "kr_vjp")
    return out, R


# Directions per launch of the second-derivative kernels: bounds their per-direction
# workspace (coefficients with tangents, about 1.6 KB per (direction, slowness, interface)).
_HVP_WS_MAX = 1 << 30


def _dir_chunks(per_dir_bytes: int, n_dir: int) -> int:
    return max(1, min(n_dir, _HVP_WS_MAX // max(per_dir_bytes, 1)))


def misfit_hvp(layers: torch.Tensor, p, omega, R_obs, V, free_surface: bool = False):
    """Exact H V of chi = sum |R - R_obs|^2 for directions V [n_dir, 4L]: ``kr_misfit_hvp``.

    Returns HV [n_dir, 4L] float64 on the device (theta order of ``jacobian``).
    """
    dev = layers.device
    L = layers.shape[1]
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    Ro = _dev_c128(R_obs, dev).reshape(n_p, n_w).contiguous()
    Vt = _dev_f64(V, dev).reshape(-1, 4 * L).contiguous()
    n_dir = Vt.shape[0]
    out = torch.empty((n_dir, 4 * L), dtype=torch.float64, device=dev)
    h = _lib.lib()
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    one = h.kr_misfit_hvp_workspace_bytes(L, n_p, n_w, 1)
    step = _dir_chunks(one, n_dir)
    for d0 in range(0, n_dir, step):
        nd = min(step, n_dir - d0)
        ws_bytes = h.kr_misfit_hvp_workspace_bytes(L, n_p, n_w, nd)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        st = h.kr_misfit_hvp(layers.data_ptr(), L, p_t.data_ptr(), n_p, w_t.data_ptr(), n_w, flags,
                             Ro.data_ptr(), Vt[d0:].data_ptr(), nd, out[d0:].data_ptr(),
                             ws.data_ptr(), ws_bytes, stream_handle(dev))
        _lib.check(st, "kr_misfit_hvp")
    return out


def jacobian_dot(layers: torch.Tensor, p, omega, V, free_surface: bool = False):
    """d/dv of the Jacobian for directions V [n_dir, 4L]: ``kr_jacobian_dot``.

    Returns Jdot [n_dir, n_p, 4L, n_w] complex128 on the device.
    """
    dev = layers.device
    L = layers.shape[1]
    p_t = _dev_f64(p, dev).reshape(-1)
    w_t = _dev_c128(omega, dev).reshape(-1)
    n_p, n_w = p_t.numel(), w_t.numel()
    Vt = _dev_f64(V, dev).reshape(-1, 4 * L).contiguous()
    n_dir = Vt.shape[0]
    out = torch.empty((n_dir, n_p, 4 * L, n_w), dtype=torch.complex128, device=dev)
    h = _lib.lib()
    flags = _lib.KR_FREE_SURFACE if free_surface else 0
    one = h.kr_jacobian_dot_workspace_bytes(L, n_p, n_w, 1)
    step = _dir_chunks(one, n_dir)
    for d0 in range(0, n_dir, step):
        nd = min(step, n_dir - d0)
        ws_bytes = h.kr_jacobian_dot_workspace_bytes(L, n_p, n_w, nd)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        st = h.kr_jacobian_dot(layers.data_ptr(), L, p_t.data_ptr(), n_p, w_t.data_ptr(), n_w,
                               flags, Vt[d0:].data_ptr(), nd, out[d0:].data_ptr(), ws.data_ptr(),
                               ws_bytes, stream_handle(dev))
        _lib.check(st, "kr_jacobian_dot")
    return out


def table_from_tensors(alpha, beta, rho, thickness, Q_alpha, Q_beta, device) -> torch.Tensor:
    """Layer table [6, L] on the device from six 1-D tensors (values only, no autograd)."""
    rows = [torch.as_tensor(x).detach().to(device=device, dtype=torch.float64).reshape(-1)
            for x in (alpha, beta, rho, thickness, Q_alpha, Q_beta)]
    L = rows[0].numel()
    if any(r.numel() != L for r in rows):
        raise ValueError("alpha, beta, rho, thickness, Q_alpha, Q_beta must have equal length")
    tab = torch.stack(rows).contiguous()
    validate_table(tab.cpu().numpy())
    return tab
