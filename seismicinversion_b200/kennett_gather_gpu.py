"""Drop-in for ``Kennett_Reflectivity.kennett_gather_gpu`` (``kennett_gather_gpu.py:56-284``).

All three stages run on the GPU in float64 with device-resident intermediates:
(1) the reflectivity grid at damped frequencies (fused Kennett kernel), (2) the
Bessel-weighted slowness sum with J0 evaluated in the kernel, (3) the Hermitian
omega -> t transform (cuFFT) with the exp(-gamma t) compensation.  The reference does (1) in
NumPy on the CPU, J0 in SciPy on the CPU and the sum in float32 on the device.
"""

from __future__ import annotations

import threading

import numpy as np
import torch

from . import device as _dev
from .earth_models import default_ocean_crust_model
from .layer_model import LayerModel, pack_layers
from .source import ricker_spectrum

__all__ = ["compute_gather_gpu", "default_ocean_crust_model", "gather_device", "save_gather_npz"]


def _gpu_bessel_summation(R, p_samples, omega_real, offsets, dp, device=None):
    """U[r, w] = dp sum_j R[j, w] taper_j p_j w J0(w p_j r) (``kennett_gather_gpu.py:56-166``).

    The Hann taper uses p_max = p_samples[-1] as in the reference.  float64 throughout.
    """
    on_device = isinstance(R, torch.Tensor) and R.is_cuda
    dev = _dev.require_cuda(R.device if on_device else device)
    p = np.asarray(p_samples.cpu() if isinstance(p_samples, torch.Tensor) else p_samples,
                   dtype=np.float64)
    taper = 0.5 * (1.0 + np.cos(np.pi * p / p[-1]))
    Rt = R if on_device else torch.as_tensor(np.ascontiguousarray(R, dtype=np.complex128), device=dev)
    U = _dev.bessel_sum(Rt, p, taper * p, dp, omega_real, offsets)
    return U if on_device else U.cpu().numpy()


def gather_device(model: LayerModel, offsets, T=64.0, nw=2048, np_slow=4096, p_max=1.2,
                  gamma=None, source_func=None, free_surface=False, device=None):
    """Device-resident gather: returns ``(time, R, U, gather)`` with R, U, gather CUDA tensors."""
    dev = _dev.require_cuda(device)
    if gamma is None:
        gamma = np.pi / T
    dw = 2.0 * np.pi / T
    omega = np.arange(1, nw, dtype=np.float64) * dw
    wmax = nw * dw
    S = ricker_spectrum(omega, wmax) if source_func is None else source_func(omega, wmax)
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    dp = p_max / np_slow
    p = np.arange(1, np_slow + 1, dtype=np.float64) * dp
    taper = 0.5 * (1.0 + np.cos(np.pi * p / p_max))
    tab = _dev.layer_table(model, dev)
    R = _dev.reflectivity(tab, p, omega + 1j * gamma, free_surface)
    U = _dev.bessel_sum(R, p, taper * p, dp, omega, offsets)
    g = _dev.traces(U, nw, S=np.asarray(S, dtype=np.complex128), decay=np.exp(-gamma * time))
    return time, R, U, g


_PINNED: dict = {}


def _pinned(shape, dtype) -> torch.Tensor:
    """A reusable page-locked host buffer (fast, async-capable device-to-host copies)."""
    key = (tuple(shape), dtype)
    buf = _PINNED.get(key)
    if buf is None:
        buf = torch.empty(shape, dtype=dtype, pin_memory=True)
        _PINNED[key] = buf
    return buf


_GRID_CACHE: dict = {}


def _grid_inputs(T, nw, np_slow, p_max, gamma, source_func, offsets_bytes):
    """Host arrays that depend only on the grid (slownesses, taper, frequencies, source
    spectrum, offsets, decay), laid out as the staging buffer holds them after a layer-table
    slot of KR_MAX_LAYERS layers.  Cached per grid: repeated gathers on one grid only pack
    their layer table.  Returns (time, dp, section offsets, section sizes, packed arrays)."""
    key = (T, nw, np_slow, p_max, gamma, source_func, offsets_bytes)
    hit = _GRID_CACHE.get(key)
    if hit is not None:
        return hit
    dw = 2.0 * np.pi / T
    omega = np.arange(1, nw, dtype=np.float64) * dw
    wmax = nw * dw
    S = ricker_spectrum(omega, wmax) if source_func is None else source_func(omega, wmax)
    nt = 2 * nw
    time = np.arange(nt, dtype=np.float64) * (T / float(nt))
    dp = p_max / np_slow
    p = np.arange(1, np_slow + 1, dtype=np.float64) * dp
    taper = 0.5 * (1.0 + np.cos(np.pi * p / p_max))
    parts = [p, taper * p, omega, omega, np.full(nw - 1, gamma),
             np.frombuffer(offsets_bytes, dtype=np.float64),
             np.asarray(S, dtype=np.complex128).view(np.float64), np.exp(-gamma * time)]
    sizes = [6 * 256] + [x.size for x in parts]
    off = np.concatenate([[0], np.cumsum([(n + 1) // 2 * 2 for n in sizes])])  # 16-B aligned
    static = np.zeros(int(off[-1] - off[1]))
    for x, a in zip(parts, off[1:-1]):
        static[a - off[1]:a - off[1] + x.size] = x
    if len(_GRID_CACHE) >= 8:
        _GRID_CACHE.pop(next(iter(_GRID_CACHE)))
    _GRID_CACHE[key] = (time, dp, off, sizes, static)
    return _GRID_CACHE[key]


def _enqueue_gather(dev, stage, off, sizes, L, nwm, nw, np_slow, dp, free_surface,
                    return_reflectivity, copy_chunks):
    """Enqueues one gather on the current stream (and the copy stream): upload of the pinned
    staging buffer, the reflectivity grid in slowness blocks with each block's host copy,
    the Bessel sum, the traces and (with the reflectivity) their host copy.  No
    synchronisation; returns (pinned host gather or None, pinned host R or None, device R,
    device gather)."""
    main = torch.cuda.current_stream(dev)
    dbuf = torch.empty(stage.shape, dtype=torch.float64, device=dev)
    dbuf.copy_(stage, non_blocking=True)
    seg = [dbuf[a:a + n] for a, n in zip(off[:-1], sizes)]
    tab = seg[0][:6 * L].view(6, L)
    p_t, pw_t = seg[1], seg[2]
    w_t = torch.complex(seg[4], seg[5])  # omega + i gamma
    wr_t, off_t = seg[3], seg[6]
    S_t = torch.view_as_complex(seg[7].view(nwm, 2))
    dec_t = seg[8]
    R = torch.empty((np_slow, nwm), dtype=torch.complex128, device=dev)
    Rh = _pinned((np_slow, nwm), torch.complex128) if return_reflectivity else None
    copy = _copy_stream(dev) if return_reflectivity else None
    n_chunks = max(1, min(copy_chunks, np_slow)) if return_reflectivity else 1
    bounds = np.linspace(0, np_slow, n_chunks + 1).astype(int)
    for a, b in zip(bounds[:-1], bounds[1:]):
        _dev.reflectivity(tab, p_t[a:b], w_t, free_surface, out=R[a:b])
        if return_reflectivity:
            ev = torch.cuda.Event()
            ev.record(main)
            copy.wait_event(ev)
            with torch.cuda.stream(copy):
                Rh[a:b].copy_(R[a:b], non_blocking=True)
    U = _dev.bessel_sum(R, p_t, pw_t, dp, wr_t, off_t)
    g = _dev.traces(U, nw, S=S_t, decay=dec_t)
    gh = None
    if return_reflectivity:
        gh = _pinned(tuple(g.shape), g.dtype)
        gh.copy_(g, non_blocking=True)
    return gh, Rh, R, g


# Gathers replayed from CUDA graphs, keyed by grid, layer count and options: a repeated call
# packs its layer table into the pinned staging buffer and replays one graph, instead of
# ~15 launches and their host-side preparation.  A key is captured on its second call (the
# first one runs eagerly and creates the cuFFT plan and kernel attributes the capture needs).
_GRAPHS: dict = {}
_GRAPH_SEEN: dict = {}
_GRAPH_MAX = 2  # each graph holds its own R grid and workspaces on the device


def _gather_graph(key, dev, enqueue_args, copy):
    hit = _GRAPHS.get(key)
    if hit is not None:
        return hit
    if key not in _GRAPH_SEEN:
        if len(_GRAPH_SEEN) >= 64:
            _GRAPH_SEEN.clear()
        _GRAPH_SEEN[key] = True
        return None
    while len(_GRAPHS) >= _GRAPH_MAX:
        _GRAPHS.pop(next(iter(_GRAPHS)))
    torch.cuda.current_stream(dev).synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, capture_error_mode="relaxed"):
        outs = _enqueue_gather(dev, *enqueue_args)
        if copy is not None:
            torch.cuda.current_stream(dev).wait_stream(copy)
    _GRAPHS[key] = (graph, outs)
    return _GRAPHS[key]


def compute_gather_gpu(model: LayerModel, offsets, T: float = 64.0, nw: int = 2048,
                       np_slow: int = 4096, p_max: float = 1.2, gamma=None, source_func=None,
                       free_surface: bool = False, device=None,
                       return_reflectivity: bool = False, copy_chunks: int = 2,
                       use_graph: bool = True, copy_outputs: bool = True):
    """``(time, offsets, gather)`` exactly as ``compute_gather_gpu`` (``kennett_gather_gpu.py:169-284``).

    With ``return_reflectivity=True`` the full R(p, omega + i gamma) grid is returned as a
    fourth element.  The grid is computed in ``copy_chunks`` slowness blocks and each block is
    copied to a pinned host buffer on a second stream while the later blocks and the Bessel
    sum run, so the host copy overlaps the compute (two blocks hide the 268 MB copy of the
    8192 x 2047 grid at ~57 GB/s; more blocks shorten the launches below full waves).
    With ``use_graph`` a grid seen before (same sizes, offsets, source, layer count and
    options) replays a captured CUDA graph.  Every returned array is the caller's own, as in
    the reference (without the R grid, the gather is a new page-locked host block that the
    device copies into directly).  With ``return_reflectivity``, ``copy_outputs=False``
    instead returns the gather and the R grid as views of this module's pinned receive
    buffers (no host copy of the 268 MB grid on the 8192 x 2047 workload), valid until the
    next call with the same grid overwrites them.  Calls share module-level staging buffers,
    grid caches and graphs under one lock: calls from several threads run one at a time.
    """
    with _CALL_LOCK:
        return _compute_gather_gpu(model, offsets, T, nw, np_slow, p_max, gamma, source_func,
                                   free_surface, device, return_reflectivity, copy_chunks,
                                   use_graph, copy_outputs)


_CALL_LOCK = threading.RLock()


def _compute_gather_gpu(model, offsets, T, nw, np_slow, p_max, gamma, source_func,
                        free_surface, device, return_reflectivity, copy_chunks, use_graph,
                        copy_outputs):
    dev = _dev.require_cuda(device)
    if gamma is None:
        gamma = np.pi / T
    tab_h = pack_layers(model)
    _dev.validate_table(tab_h)
    offsets_h = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1)
    nwm, L = nw - 1, tab_h.shape[1]
    grid_key = (float(T), int(nw), int(np_slow), float(p_max), float(gamma), source_func,
                offsets_h.tobytes())
    time, dp, off, sizes, static = _grid_inputs(*grid_key)
    main = torch.cuda.current_stream(dev)
    # every input in one pinned staging buffer and one upload ahead of the first kernel, so
    # that the kernels run back to back without host round trips between them; on a grid
    # seen before only the layer table is packed
    stage = _pinned((int(off[-1]),), torch.float64)
    sn = stage.numpy()
    sn[off[1]:] = static
    sn[:tab_h.size] = tab_h.ravel()
    args = (stage, off, sizes, L, nwm, nw, int(np_slow), dp, bool(free_surface),
            bool(return_reflectivity), int(copy_chunks))
    copy = _copy_stream(dev) if return_reflectivity else None
    entry = None
    if use_graph:
        entry = _gather_graph((dev, grid_key) + args[3:], dev, args, copy)
    if entry is not None:
        graph, (gh, Rh, _, g) = entry
        graph.replay()
    else:
        gh, Rh, R, g = _enqueue_gather(dev, *args)
        if return_reflectivity:
            R.record_stream(copy)
    if return_reflectivity:
        copy.synchronize()
        main.synchronize()
        Rn, gn = Rh.numpy(), gh.numpy()
        if copy_outputs:
            Rn, gn = Rn.copy(), gn.copy()
        return time.copy(), np.asarray(offsets), gn, Rn
    # the traces go straight into a new page-locked block from torch's caching host allocator:
    # the caller's own array, no host-side copy (freed blocks are reused without new faults)
    out = torch.empty(tuple(g.shape), dtype=g.dtype, pin_memory=True)
    out.copy_(g, non_blocking=True)
    main.synchronize()
    return time.copy(), np.asarray(offsets), out.numpy()


_COPY_STREAMS: dict = {}


def _copy_stream(dev) -> torch.cuda.Stream:
    s = _COPY_STREAMS.get(dev)
    if s is None:
        s = torch.cuda.Stream(dev)
        _COPY_STREAMS[dev] = s
    return s


def save_gather_npz(path, time, offsets, gather):
    """Write a gather as ``.npz`` with keys ``time``, ``offsets``, ``gather`` -- the file the
    reference CLI writes (``kennett_gather_gpu.py:429-436``).  Returns the path written."""
    from pathlib import Path

    out = Path(path).with_suffix(".npz")
    np.savez(out, time=np.asarray(time), offsets=np.asarray(offsets), gather=np.asarray(gather))
    return out


def main(argv=None) -> None:
    """Command line as ``python -m Kennett_Reflectivity.kennett_gather_gpu``
    (``kennett_gather_gpu.py:287-436``): default 5-layer model, writes ``<output>.npz``.
    Plotting is not provided (the reference skips it too when matplotlib is missing)."""
    import argparse
    import logging

    ap = argparse.ArgumentParser(description="Seismogram gather via Kennett reflectivity (B200).")
    ap.add_argument("--r-min", type=float, default=0.5)
    ap.add_argument("--r-max", type=float, default=50.0)
    ap.add_argument("--dr", type=float, default=0.5)
    ap.add_argument("-T", "--duration", type=float, default=64.0)
    ap.add_argument("-n", "--nw", type=int, default=2048)
    ap.add_argument("--np", dest="np_slow", type=int, default=4096)
    ap.add_argument("--p-max", type=float, default=1.2)
    ap.add_argument("--gamma", type=float, default=None)
    ap.add_argument("--t-max", type=float, default=30.0)
    ap.add_argument("-o", "--output", default="gather_gpu.png")
    ap.add_argument("--no-plot", action="store_true")
    ap.add_argument("--free-surface", action="store_true")
    ap.add_argument("--device", default=None)
    args = ap.parse_args(argv)
    offsets = np.arange(args.r_min, args.r_max + args.dr / 2, args.dr)
    device = args.device if args.device not in (None, "mps", "cpu") else None
    time, offs, gather = compute_gather_gpu(default_ocean_crust_model(), offsets, T=args.duration,
                                            nw=args.nw, np_slow=args.np_slow, p_max=args.p_max,
                                            gamma=args.gamma, free_surface=args.free_surface,
                                            device=device)
    if not args.no_plot:
        logging.getLogger(__name__).warning("plotting is not provided; writing data only")
    out = save_gather_npz(args.output, time, offs, gather)
    logging.getLogger(__name__).info("Data saved to %s", out)


if __name__ == "__main__":
    main()
