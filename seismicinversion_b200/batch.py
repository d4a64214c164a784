"""Batched evaluation of many earth models of uneven size (``kr_batch_*``).

A ``ModelBatch`` packs models with different layer counts, slowness and frequency grids
into device buffers, plans the batch once (work lists sorted by cost), and runs it as a
persistent launch: forward R grids for some models, forward + misfit gradient for others.
The launch needs no host synchronisation or allocation, so it can be captured in a CUDA
graph and replayed; ``update_layers`` changes parameter values in place between replays
(inversion iterates of the same shapes).

The schedule (threads per block, frequencies per work item) is chosen by ``autotune``, which
times the candidate schedules on the batch itself and caches the winner per batch signature.
"""

from __future__ import annotations

import ctypes
import json
import os
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib
from . import device as D
from .layer_model import LayerModel, pack_layers

__all__ = ["BatchItem", "ModelBatch", "autotune", "SCHEDULES"]

#: Candidate schedules: (threads per block, frequencies per work item).  32 threads is the
#: warp-per-pair schedule: one warp owns a (model, slowness) pair's frequency range.
SCHEDULES = [(32, 64), (32, 128), (64, 64), (64, 128), (128, 128), (128, 256), (128, 512),
             (64, 256), (128, 1024), (128, 2048)]


@dataclass
class BatchItem:
    """One model of a batch.

    ``gradient=True`` asks for chi = sum |R - R_obs|^2 and its gradient with respect to every
    layer's (alpha, beta, rho, h) (``R_obs`` required, shape (n_p, n_w)); otherwise the R grid
    is computed.  ``store_R`` also stores R for gradient models.
    """

    model: LayerModel
    p: np.ndarray
    omega: np.ndarray
    gradient: bool = False
    R_obs: np.ndarray | None = None
    free_surface: bool = False
    store_R: bool = False


def _flat(x, dtype) -> torch.Tensor:
    """1-D tensor view of x (numpy or torch, host or device) in the given dtype."""
    if isinstance(x, torch.Tensor):
        return x.detach().to(dtype).reshape(-1)
    return torch.as_tensor(np.ascontiguousarray(x)).to(dtype).reshape(-1)


def _cat_into(out: torch.Tensor, parts):
    """Concatenate 1-D parts into the device view ``out`` (one kernel for device parts).
    Returns the pinned host staging tensor when some part lives on the host (the caller
    keeps it until the stream-ordered copy has run), else None."""
    if not parts:
        return None
    n = sum(t.numel() for t in parts)
    if all(t.is_cuda for t in parts):
        torch.cat([t.to(out.dtype) for t in parts], out=out[:n])
        return None
    host = torch.cat([t.cpu().to(out.dtype) for t in parts]).pin_memory()
    out[:n].copy_(host, non_blocking=True)
    return host


def _size_class(nbytes: int) -> int:
    """Allocation size for a batch block: four classes per power of two (multiples of a
    quarter of the power of two below: at most 25 % slack), at least 1 MiB, so that batches of
    similar size reuse the same cached blocks."""
    nbytes = max(int(nbytes), 1 << 20)
    step = 1 << max(0, (nbytes - 1).bit_length() - 3)
    return (nbytes + step - 1) // step * step


class ModelBatch:
    """Device-resident packed batch with its plan; see the module docstring.

    ``p``, ``omega`` and ``R_obs`` of the items may be NumPy arrays or (CUDA) tensors; device
    tensors are concatenated on the device without a host round trip.  ``alloc_stream``: take
    the batch's device block from that stream's allocator pool (a server running batches on
    several streams then keeps one pool of cached blocks instead of one per stream)."""

    def __init__(self, items: list[BatchItem], schedule: tuple[int, int] | None = None,
                 device=None, alloc_stream: torch.cuda.Stream | None = None):
        self.dev = D.require_cuda(device)
        self.items = items
        n = len(items)
        desc = np.zeros(n, dtype=_lib.MODEL_DESC_FIELDS)
        tabs, ps, ws, obs = [], [], [], []
        lo = po = wo = ro = oo = go = 0
        self.max_layers = 2
        # items passing the very same p / omega / R_obs object share one device copy
        seen_p, seen_w, seen_o = {}, {}, {}
        for b, it in enumerate(items):
            tab = pack_layers(it.model)
            D.validate_table(tab)
            L = tab.shape[1]
            p = _flat(it.p, torch.float64)
            w = _flat(it.omega, torch.complex128)
            n_p, n_w = p.numel(), w.numel()
            flags = _lib.KR_FREE_SURFACE if it.free_surface else 0
            if it.gradient:
                if it.R_obs is None:
                    raise ValueError(f"batch item {b}: gradient requested without R_obs")
                flags |= _lib.KR_BATCH_GRADIENT | (_lib.KR_BATCH_STORE_R if it.store_R else 0)
            d = desc[b]
            d["n_layers"], d["n_p"], d["n_w"], d["flags"] = L, n_p, n_w, flags
            d["layers_off"] = lo
            tabs.append(tab.ravel())
            lo += tab.size
            if id(it.p) in seen_p:
                d["p_off"] = seen_p[id(it.p)]
            else:
                d["p_off"] = seen_p[id(it.p)] = po
                ps.append(p)
                po += n_p
            if id(it.omega) in seen_w:
                d["omega_off"] = seen_w[id(it.omega)]
            else:
                d["omega_off"] = seen_w[id(it.omega)] = wo
                ws.append(w)
                wo += n_w
            if (not it.gradient) or it.store_R:
                d["R_off"] = ro
                ro += n_p * n_w
            if it.gradient:
                if id(it.R_obs) in seen_o:
                    d["obs_off"] = seen_o[id(it.R_obs)]
                else:
                    o = _flat(it.R_obs, torch.complex128)
                    if o.numel() != n_p * n_w:
                        raise ValueError(f"batch item {b}: R_obs must have shape ({n_p}, {n_w})")
                    d["obs_off"] = seen_o[id(it.R_obs)] = oo
                    obs.append(o)
                    oo += o.numel()
                d["grad_off"] = go
                go += 4 * L + 1
            self.max_layers = max(self.max_layers, L)
        self.desc = desc
        self.graph = None
        self.schedule = None
        self.plan = None
        schedule = tuple(schedule or (128, 256))
        plan_bytes = self._plan_bytes(schedule)
        # One device block per batch holds every buffer (layers, grids, R_obs, R, chi_grad,
        # plan), its size rounded up to a size class: a stream of batches of varying shape
        # then reuses cached blocks of a few classes instead of calling cudaMalloc (slow, and
        # able to stall the host for tens of ms) for each of several buffers per batch.
        sizes = [8 * max(lo, 1), 8 * max(po, 1), 16 * max(wo, 1), 16 * max(oo, 1),
                 16 * max(ro, 1), 8 * max(go, 1), plan_bytes]
        offs, total = [], 0
        for n_b in sizes:
            offs.append(total)
            total += (n_b + 255) // 256 * 256
        if alloc_stream is None:
            block = torch.empty(_size_class(total), dtype=torch.uint8, device=self.dev)
        else:
            # allocated from one stream's pool (shared by every batch of a server, whatever
            # stream runs it) and marked as used by the stream that runs this batch
            with torch.cuda.stream(alloc_stream):
                block = torch.empty(_size_class(total), dtype=torch.uint8, device=self.dev)
            block.record_stream(torch.cuda.current_stream(self.dev))
        view = [block[o:o + n_b] for o, n_b in zip(offs, sizes)]
        self.layers = view[0].view(torch.float64)
        staged = torch.from_numpy(np.concatenate(tabs) if tabs else np.zeros(1)).pin_memory()
        self.layers.copy_(staged, non_blocking=True)
        self.p = view[1].view(torch.float64)
        self.omega = view[2].view(torch.complex128)
        self.R_obs = view[3].view(torch.complex128) if obs else None
        # pinned sources stay referenced until their stream-ordered copies have run
        self._staged = [staged, _cat_into(self.p, ps), _cat_into(self.omega, ws),
                        _cat_into(self.R_obs, obs) if obs else None]
        self.R = view[4].view(torch.complex128)
        self.chi_grad = view[5].view(torch.float64)
        self.chi_grad.zero_()
        self._block = block
        self.set_schedule(schedule, plan=view[6])

    @classmethod
    def from_tables(cls, tables: np.ndarray, p, omega, free_surface: bool = False,
                    schedule: tuple[int, int] | None = None, device=None) -> "ModelBatch":
        """Forward batch of same-shape models from layer tables [n, 6, L] on one shared
        slowness / frequency grid (vectorised packing; R of model b is
        ``R[b*n_p*n_w:(b+1)*n_p*n_w]``)."""
        tables = np.ascontiguousarray(tables, dtype=np.float64)
        n, six, L = tables.shape
        if six != 6:
            raise ValueError("tables must have shape [n, 6, n_layers]")
        for b in range(n):
            D.validate_table(tables[b])
        p = np.ascontiguousarray(p, dtype=np.float64).reshape(-1)
        w = np.ascontiguousarray(omega, dtype=np.complex128).reshape(-1)
        self = cls.__new__(cls)
        self.dev = D.require_cuda(device)
        self.items = None
        desc = np.zeros(n, dtype=_lib.MODEL_DESC_FIELDS)
        desc["n_layers"], desc["n_p"], desc["n_w"] = L, len(p), len(w)
        desc["flags"] = _lib.KR_FREE_SURFACE if free_surface else 0
        desc["layers_off"] = np.arange(n) * 6 * L
        desc["R_off"] = np.arange(n) * len(p) * len(w)
        self.desc = desc
        self.max_layers = L
        self.layers = torch.as_tensor(tables.reshape(-1), device=self.dev)
        self.p = torch.as_tensor(p, device=self.dev)
        self.omega = torch.as_tensor(w, device=self.dev)
        self.R_obs = None
        self.R = torch.empty(max(n * len(p) * len(w), 1), dtype=torch.complex128, device=self.dev)
        self.chi_grad = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.graph = None
        self.schedule = None
        self.plan = None
        self.set_schedule(schedule or (128, 128))
        return self

    # -- planning ------------------------------------------------------------------------
    def _cfg(self, schedule):
        return _lib.BatchConfig(int(schedule[0]), int(schedule[1]), 0, 0)

    def _plan_bytes(self, schedule) -> int:
        h = _lib.lib()
        cfg = self._cfg(schedule)
        nbytes = h.kr_batch_plan_bytes(self.desc.ctypes.data, len(self.desc), ctypes.byref(cfg))
        if nbytes == 0:
            raise ValueError(f"invalid batch or schedule {schedule}")
        return int(nbytes)

    def set_schedule(self, schedule: tuple[int, int], plan: torch.Tensor | None = None) -> None:
        """(Re)plan the batch for a schedule (threads, frequencies per item)."""
        h = _lib.lib()
        cfg = self._cfg(schedule)
        n = len(self.desc)
        nbytes = self._plan_bytes(schedule)
        meta = h.kr_batch_plan_meta_bytes(self.desc.ctypes.data, n, ctypes.byref(cfg))
        image = torch.empty(meta, dtype=torch.uint8, pin_memory=True)
        st = h.kr_batch_plan_host(self.desc.ctypes.data, n, ctypes.byref(cfg), image.data_ptr(),
                                  meta)
        _lib.check(st, "kr_batch_plan_host")
        if plan is None or plan.numel() < nbytes:
            plan = torch.empty(nbytes, dtype=torch.uint8, device=self.dev)
        plan[:meta].copy_(image, non_blocking=True)  # stream-ordered before any launch
        self._plan_image = image  # keep the pinned source alive until the copy has run
        self.plan, self.schedule, self._cfg_obj, self.graph = plan, tuple(schedule), cfg, None

    # -- running -------------------------------------------------------------------------
    def launch(self) -> None:
        """Enqueue the batch on the current stream (no synchronisation)."""
        h = _lib.lib()
        obs = self.R_obs.data_ptr() if self.R_obs is not None else None
        st = h.kr_batch_launch(self.plan.data_ptr(), ctypes.byref(self._cfg_obj), self.max_layers,
                               self.layers.data_ptr(), self.p.data_ptr(), self.omega.data_ptr(),
                               obs, self.R.data_ptr(), self.chi_grad.data_ptr(),
                               D.stream_handle(self.dev))
        _lib.check(st, "kr_batch_launch")

    def capture(self) -> torch.cuda.CUDAGraph:
        """Capture one launch in a CUDA graph (replay with ``run``)."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.launch()  # warm: loads modules outside capture
        torch.cuda.current_stream(self.dev).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.launch()
        self.graph = g
        return g

    def run(self) -> None:
        """Replay the captured graph if any, else launch directly."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self.launch()

    def update_layers(self, models: list[LayerModel]) -> None:
        """Copy new layer values (same layer counts) into the device buffer in place."""
        tabs = []
        for b, m in enumerate(models):
            tab = pack_layers(m)
            if tab.shape[1] != self.desc[b]["n_layers"]:
                raise ValueError(f"model {b}: layer count changed")
            D.validate_table(tab)
            tabs.append(tab.ravel())
        self.layers.copy_(torch.from_numpy(np.concatenate(tabs)), non_blocking=False)

    # -- results -------------------------------------------------------------------------
    def reflectivity(self, b: int) -> torch.Tensor:
        """R grid (n_p, n_w) of model b (device view)."""
        d = self.desc[b]
        if (d["flags"] & _lib.KR_BATCH_GRADIENT) and not (d["flags"] & _lib.KR_BATCH_STORE_R):
            raise ValueError(f"model {b} is a gradient model without store_R")
        n = int(d["n_p"]) * int(d["n_w"])
        return self.R[int(d["R_off"]):int(d["R_off"]) + n].view(int(d["n_p"]), int(d["n_w"]))

    def misfit_gradient(self, b: int) -> tuple[torch.Tensor, torch.Tensor]:
        """(chi, gradient [4L]) of gradient model b (device views)."""
        d = self.desc[b]
        if not d["flags"] & _lib.KR_BATCH_GRADIENT:
            raise ValueError(f"model {b} is not a gradient model")
        L = int(d["n_layers"])
        v = self.chi_grad[int(d["grad_off"]):int(d["grad_off"]) + 4 * L + 1]
        return v[4 * L], v[:4 * L]

    def work(self) -> dict:
        """Algorithmic work of one launch: forward and gradient (omega, p, interface) updates."""
        fwd = grad = 0
        for d in self.desc:
            u = int(d["n_p"]) * int(d["n_w"]) * (int(d["n_layers"]) - 1)
            if d["flags"] & _lib.KR_BATCH_GRADIENT:
                grad += u
            else:
                fwd += u
        return {"forward_updates": fwd, "gradient_updates": grad,
                "gradient_models": int(np.sum(self.desc["flags"] & _lib.KR_BATCH_GRADIENT > 0)),
                "models": len(self.desc)}

    def signature(self) -> str:
        w = self.work()
        Ls = self.desc["n_layers"]
        return (f"m{len(self.desc)}-f{w['forward_updates']:.2e}-g{w['gradient_updates']:.2e}"
                f"-L{int(Ls.min())}-{int(Ls.max())}")


def _time_launch(batch: ModelBatch, reps: int) -> float:
    st = torch.cuda.current_stream(batch.dev)
    batch.launch()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        batch.launch()
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b) / reps


_TUNE_CACHE: dict = {}


def autotune(batch: ModelBatch, candidates=None, reps: int = 2, cache_file: str | None = None):
    """Time each candidate schedule on ``batch`` and keep the fastest.

    Returns ``(best_schedule, {schedule: ms})``.  Winners are cached per batch signature in
    memory and, if ``cache_file`` (or ``KR_TUNE_CACHE``) names a JSON file, on disk.
    """
    sig = batch.signature()
    path = cache_file or os.environ.get("KR_TUNE_CACHE")
    disk = {}
    if path and Path(path).exists():
        try:
            disk = json.loads(Path(path).read_text())
        except (OSError, ValueError):
            disk = {}
    hit = _TUNE_CACHE.get(sig) or disk.get(sig)
    if hit:
        batch.set_schedule(tuple(hit))
        return tuple(hit), {}
    times = {}
    for sch in candidates or SCHEDULES:
        batch.set_schedule(sch)
        times[sch] = _time_launch(batch, reps)
    best = min(times, key=times.get)
    batch.set_schedule(best)
    _TUNE_CACHE[sig] = list(best)
    if path:
        disk[sig] = list(best)
        try:
            Path(path).write_text(json.dumps(disk, indent=1))
        except OSError:
            pass
    return best, times


def per_call_reference(items: list[BatchItem], device=None) -> float:
    """Wall time (s) of the plain per-call path: one fused-kernel call per model with a
    synchronisation after each (kr_reflectivity or kr_misfit_gradient), for comparison."""
    dev = D.require_cuda(device)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for it in items:
        tab = D.layer_table(it.model, dev)
        if it.gradient:
            D.misfit_gradient(tab, it.p, it.omega, it.R_obs, it.free_surface)
        else:
            D.reflectivity(tab, it.p, it.omega, it.free_surface)
        torch.cuda.synchronize(dev)
    return time.perf_counter() - t0
