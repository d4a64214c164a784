"""Continuous-batching request loop for forward and forward+gradient solves.

Clients ``submit`` requests of any size (a model, its slowness and frequency grids, and for
gradient requests the observed R) from any thread; each returns a ``Request`` whose
``done`` event is the host-visible completion flag.  A scheduler thread:

* admits pending requests in arrival order while the device-memory footprint of everything
  admitted stays within ``hbm_budget_bytes`` and the batch has free slots
  (``max_batch_requests``); a request that can never fit is rejected, one that cannot fit
  *now* waits (no request is dropped silently);
* launches each admitted group as one persistent batched launch (``ModelBatch``) on one of
  ``n_streams`` streams, keeping up to ``max_inflight`` batches on the GPU at once, so
  requests that arrive while others run are batched into the next launch and their work
  overlaps on the device; a group of up to four requests (a lightly or moderately loaded
  server) runs the single-model kernels instead, which skip the batch machinery;
* polls completion events and marks requests done.  Results stay on the device as tensors
  (views of the batch's single device block), so the budget keeps a batch's bytes charged
  until every request of that batch has released its results: ``Request.release()``, or
  garbage collection of the request together with every result tensor it handed out.  A
  client that keeps results resident therefore holds budget, exactly as it holds HBM.

The executor is pluggable (``executor=``); the default runs ``ModelBatch`` on the GPU.
Latency is measured from ``submit`` to the moment the scheduler sets ``done``.
"""

from __future__ import annotations

import collections
import threading
import time
import weakref
from dataclasses import dataclass, field

import numpy as np

from .layer_model import LayerModel, pack_layers

__all__ = ["Request", "KennettServer", "GpuBatchExecutor", "request_bytes",
           "RequestRejected"]


class RequestRejected(Exception):
    """The request can never be served (invalid, larger than the budget, queue full)."""


@dataclass
class Request:
    model: LayerModel
    p: np.ndarray
    omega: np.ndarray
    gradient: bool = False
    R_obs: np.ndarray | None = None
    free_surface: bool = False
    # filled by the server
    id: int = -1
    t_submit: float = 0.0
    t_admit: float = 0.0
    t_launched: float = 0.0
    t_done: float = 0.0
    nbytes: int = 0
    done: threading.Event = field(default_factory=threading.Event)
    result: dict | None = None
    error: BaseException | None = None
    cancelled: bool = False
    _lease: object = None
    _callbacks: list = field(default_factory=list)
    _cb_lock: threading.Lock = field(default_factory=threading.Lock)

    def add_done_callback(self, fn) -> None:
        """Calls ``fn(request)`` once the request is done (at once if it already is), on the
        thread that completes it."""
        with self._cb_lock:
            if not self.done.is_set():
                self._callbacks.append(fn)
                return
        fn(self)

    def _finish(self) -> None:
        with self._cb_lock:
            self.done.set()
            cbs, self._callbacks = self._callbacks, []
        for fn in cbs:
            try:
                fn(self)
            except Exception:  # a client callback must not stop the scheduler
                pass

    def wait(self, timeout: float | None = None) -> dict:
        if not self.done.wait(timeout):
            raise TimeoutError(f"request {self.id} not done after {timeout} s")
        if self.error is not None:
            raise self.error
        return self.result

    def release(self) -> None:
        """Drop this request's results.  Its batch's bytes return to the server's budget once
        every request of the batch has released them (or been collected along with the result
        tensors it handed out): the batch's results share one device block."""
        self.result = None
        self._lease = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


def request_bytes(model: LayerModel, n_p: int, n_w: int, gradient: bool) -> int:
    """Device bytes one request occupies while admitted, an upper bound: its inputs and outputs
    and its share of the batch plan (per slowness: layer terms, interface coefficients and, for
    gradients, derivative factors and coefficient tangents, each section padded to 256 B as
    the plan lays them out, plus its pair record and work items), times 1.25 for the size-class
    rounding of the batch's single device block.  Left out: that block's 1 MiB minimum, at most
    1 MiB per batch in flight."""
    L = model.n_layers
    I = L - 1

    def a256(x):
        return (x + 255) // 256 * 256

    b = 48 * L + 8 * n_p + 16 * n_w + 16 * n_p * n_w  # layers, p, omega, R
    coef = a256(96 * L) + a256(336 * I) + 256  # LayerP, Iface; pair record and work items
    if gradient:
        b += 16 * n_p * n_w + 8 * (4 * L + 1)  # R_obs, chi_grad
        coef += a256(112 * L) + a256(960 * I)  # LayerD, ScatTan
    return int(1.25 * (b + n_p * coef + 1024))


class _Lease:
    """Budget share of one completed batch: its requests' bytes return to the server when the
    last reference goes (the requests' ``_lease``, the result dicts and result tensors)."""

    def __init__(self, released: collections.deque, nbytes: int):
        self.nbytes = nbytes
        weakref.finalize(self, released.append, nbytes)


class _Result(dict):
    """A request's result dict; keeps its batch's lease alive while the client holds it."""

    __slots__ = ("_lease",)


def _attach(res, lease):
    out = _Result(res)
    out._lease = lease
    for v in res.values():
        try:  # tensors carry the lease too, so a result tensor alone keeps its bytes charged
            v._kr_lease = lease
        except AttributeError:
            pass
    return out


@dataclass
class _Record:
    """Timing record of a finished request (the server keeps these, not the requests)."""

    t_submit: float
    t_admit: float
    t_launched: float
    t_done: float
    ok: bool

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class GpuBatchExecutor:
    """Runs an admitted group as one ModelBatch launch on a stream; ``ready`` polls its event.

    Groups of at most ``direct_max_requests`` requests (default 4) run the single-model
    entry points (``kr_reflectivity``, ``kr_misfit_gradient`` with R) on the stream instead:
    the same R bit for bit, the gradient to rounding (the batch adds per-block partials in
    another order), without the plan build."""

    def __init__(self, device=None, n_streams: int = 2, schedule=(128, 256),
                 direct_max_requests: int = 4):
        import torch

        from . import device as D

        self.torch = torch
        self.D = D
        self.direct_max = int(direct_max_requests)
        self.dev = D.require_cuda(device)
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(n_streams)]
        # every batch's device block comes from this stream's allocator pool, so cached
        # blocks serve all execution streams (a pool per stream would keep calling cudaMalloc
        # for sizes that another stream has cached)
        self.alloc_stream = torch.cuda.Stream(self.dev)
        self.schedule = schedule
        self._k = 0

    def prewarm(self, device_bytes: int, host_bytes: int = 16 << 20,
                stream_bytes: int = 256 << 20) -> None:
        """Reserve a caching-allocator segment on the allocation stream (and pinned host blocks) so
        that steady-state batches reuse cached memory instead of calling cudaMalloc /
        cudaHostAlloc, which are slow and (cudaMalloc) synchronise the device.  Each execution
        stream also gets ``stream_bytes`` of large blocks and a few small-pool segments: groups
        of one request allocate their outputs and workspaces there."""
        torch = self.torch
        with torch.cuda.stream(self.alloc_stream):
            x = torch.empty(int(device_bytes), dtype=torch.uint8, device=self.dev)
            del x
        for s in self.streams:
            with torch.cuda.stream(s):
                xs = [torch.empty(int(stream_bytes), dtype=torch.uint8, device=self.dev)]
                xs += [torch.empty(512 << 10, dtype=torch.uint8, device=self.dev)
                       for _ in range(16)]
                del xs
        # one pinned block per power-of-two size class from 1 KB up (the host caching
        # allocator serves plan images and staging copies from these)
        sizes, b = [], 1024
        while b <= int(host_bytes):
            sizes.append(b)
            b *= 2
        blocks = [torch.empty(n, dtype=torch.uint8, pin_memory=True) for n in sizes for _ in range(8)]
        del blocks
        torch.cuda.synchronize(self.dev)

    def launch(self, reqs: list[Request]):
        from .batch import BatchItem, ModelBatch

        torch = self.torch
        s = self.streams[self._k % len(self.streams)]
        self._k += 1
        if len(reqs) <= self.direct_max:
            with torch.cuda.stream(s):
                res = [self._direct(r) for r in reqs]
                ev = torch.cuda.Event()
                ev.record(s)
            return (None, ev, res)
        with torch.cuda.stream(s):
            items = [BatchItem(r.model, r.p, r.omega, gradient=r.gradient, R_obs=r.R_obs,
                               free_surface=r.free_surface, store_R=r.gradient) for r in reqs]
            batch = ModelBatch(items, schedule=self.schedule, device=self.dev,
                               alloc_stream=self.alloc_stream)
            batch.launch()
            ev = torch.cuda.Event()
            ev.record(s)
        return (batch, ev, None)

    def _direct(self, r: Request) -> dict:
        D = self.D
        tab = D.layer_table(r.model, self.dev)
        if r.gradient:
            out, R = D.misfit_gradient(tab, r.p, r.omega, r.R_obs, r.free_surface, want_R=True)
            L = tab.shape[1]
            return {"R": R, "chi": out[4 * L], "grad": out[:4 * L]}
        return {"R": D.reflectivity(tab, r.p, r.omega, r.free_surface)}

    def ready(self, handle) -> bool:
        return handle[1].query()

    def results(self, handle, reqs: list[Request]) -> list[dict]:
        batch, _, direct = handle
        if direct is not None:
            return direct
        out = []
        for b, r in enumerate(reqs):
            res = {"R": batch.reflectivity(b)}
            if r.gradient:
                chi, g = batch.misfit_gradient(b)
                res["chi"], res["grad"] = chi, g
            out.append(res)
        return out


class KennettServer:
    """Continuous-batching server; see the module docstring."""

    def __init__(self, executor=None, hbm_budget_bytes: int = 120 * 10**9,
                 max_batch_requests: int = 256, max_inflight: int = 2,
                 max_pending: int = 1_000_000, poll_interval: float = 50e-6,
                 min_batch_wait: float = 0.0, prewarm_bytes: int = 0):
        """``executor``: runs admitted groups (default ``GpuBatchExecutor``).
        ``hbm_budget_bytes``: device bytes of admitted and unreleased requests (see the module
        docstring).  ``max_batch_requests``: requests per launch.  ``max_inflight``: batches on
        the GPU at once.  ``max_pending``: waiting requests before submissions are rejected.
        ``min_batch_wait``: seconds the first waiting request may wait for others when the GPU
        is idle.  ``prewarm_bytes``: device bytes to reserve in the executor's pool."""
        # one more stream than batches in flight: the stream a new batch is built on has
        # always finished its previous batch, so host-side uploads never wait on the GPU
        self.executor = (executor if executor is not None
                         else GpuBatchExecutor(n_streams=int(max_inflight) + 1))
        if prewarm_bytes and hasattr(self.executor, "prewarm"):
            self.executor.prewarm(min(int(prewarm_bytes), int(hbm_budget_bytes)))
        self.budget = int(hbm_budget_bytes)
        self.max_batch = int(max_batch_requests)
        self.max_inflight = int(max_inflight)
        self.max_pending = int(max_pending)
        self.poll = float(poll_interval)
        self.min_batch_wait = float(min_batch_wait)
        self._pending: collections.deque[Request] = collections.deque()
        self._inflight: list[tuple[object, list[Request]]] = []
        self._used = 0
        # bytes of released batches, appended by lease finalizers from any thread (a deque
        # append needs no lock) and drained by the scheduler
        self._released: collections.deque[int] = collections.deque()
        self._lock = threading.Lock()
        self._wake = threading.Condition(self._lock)
        self._stop = False
        self._next_id = 0
        self.completed: list[_Record] = []
        self.batches_launched = 0
        self.peak_bytes = 0
        self._thread = threading.Thread(target=self._loop, name="kennett-server", daemon=True)
        self._thread.start()

    # -- client side ---------------------------------------------------------------------
    def submit(self, model: LayerModel, p, omega, gradient: bool = False, R_obs=None,
               free_surface: bool = False) -> Request:
        if not hasattr(p, "is_cuda"):
            p = np.ascontiguousarray(np.atleast_1d(p), dtype=np.float64)
        if not hasattr(omega, "is_cuda"):
            omega = np.ascontiguousarray(np.atleast_1d(omega), dtype=np.complex128)
        req = Request(model, p, omega, gradient, R_obs, free_surface)
        req.t_submit = time.perf_counter()
        try:
            pack_layers(model)
            if gradient:
                if R_obs is None or tuple(R_obs.shape) != (len(p), len(omega)):
                    raise ValueError("gradient request needs R_obs of shape (n_p, n_omega)")
            if len(p) == 0 or len(omega) == 0:
                raise ValueError("empty slowness or frequency grid")
            req.nbytes = request_bytes(model, len(p), len(omega), gradient)
            if req.nbytes > self.budget:
                raise RequestRejected(f"request needs {req.nbytes} B > budget {self.budget} B")
        except (ValueError, RequestRejected) as e:
            req.error = e if isinstance(e, RequestRejected) else RequestRejected(str(e))
            req.t_done = time.perf_counter()
            req._finish()
            return req
        with self._lock:
            full = len(self._pending) >= self.max_pending
            if not full:
                req.id = self._next_id
                self._next_id += 1
                self._pending.append(req)
                self._wake.notify()
        if full:
            req.error = RequestRejected("queue full")
            req.t_done = time.perf_counter()
            req._finish()
        return req

    def cancel(self, req: Request) -> bool:
        """Cancel a request that has not been admitted yet (True if it was)."""
        with self._lock:
            if req not in self._pending:
                return False
            self._pending.remove(req)
        req.cancelled = True
        req.error = RequestRejected("cancelled")
        req.t_done = time.perf_counter()
        req._finish()
        return True

    def close(self, timeout: float = 60.0) -> None:
        with self._lock:
            self._stop = True
            self._wake.notify()
        self._thread.join(timeout)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def used_bytes(self) -> int:
        """Budget held by admitted requests whose results have not been released."""
        with self._lock:
            self._drain_released()
            return self._used

    # -- scheduler -----------------------------------------------------------------------
    def _drain_released(self) -> None:
        while self._released:
            self._used -= self._released.popleft()

    def _admit(self) -> list[Request]:
        self._drain_released()
        group: list[Request] = []
        while self._pending and len(group) < self.max_batch:
            r = self._pending[0]
            if self._used + r.nbytes > self.budget:
                break  # FIFO: wait for memory to free up
            self._pending.popleft()
            self._used += r.nbytes
            r.t_admit = time.perf_counter()
            group.append(r)
        self.peak_bytes = max(self.peak_bytes, self._used)
        return group

    def _complete(self) -> None:
        still = []
        for handle, reqs in self._inflight:
            if self.executor.ready(handle):
                try:
                    res = self.executor.results(handle, reqs)
                    err = None
                except BaseException as e:  # device-side failure reported by the library
                    res, err = [None] * len(reqs), e
                now = time.perf_counter()
                lease = None
                if err is None:
                    lease = _Lease(self._released, sum(r.nbytes for r in reqs))
                with self._lock:
                    for r, x in zip(reqs, res):
                        if err is None:
                            r.result, r._lease = _attach(x, lease), lease
                        else:
                            r.error = err
                            self._used -= r.nbytes
                        r.t_done = now
                        self.completed.append(_Record(r.t_submit, r.t_admit, r.t_launched,
                                                      r.t_done, err is None))
                for r in reqs:  # outside the lock: completion runs client callbacks
                    r._finish()
                del lease, res
            else:
                still.append((handle, reqs))
        self._inflight = still

    def _loop(self) -> None:
        while True:
            self._complete()
            with self._lock:
                if self._stop and not self._pending and not self._inflight:
                    return
                group = []
                if len(self._inflight) < self.max_inflight and self._pending:
                    if self.min_batch_wait > 0 and not self._inflight:
                        age = time.perf_counter() - self._pending[0].t_submit
                        if age < self.min_batch_wait and len(self._pending) < self.max_batch:
                            self._wake.wait(self.min_batch_wait - age)
                            continue
                    group = self._admit()
                if not group and not self._inflight and not self._stop:
                    self._wake.wait(0.01)
                    continue
            if group:
                try:
                    handle = self.executor.launch(group)
                    t_l = time.perf_counter()
                    for r in group:
                        r.t_launched = t_l
                    self._inflight.append((handle, group))
                    self.batches_launched += 1
                except BaseException as e:
                    now = time.perf_counter()
                    with self._lock:
                        for r in group:
                            r.error, r.t_done = e, now
                            self._used -= r.nbytes
                    for r in group:
                        r._finish()
            elif self._inflight:
                time.sleep(self.poll)

    # -- statistics ----------------------------------------------------------------------
    def stats(self, since: float = 0.0) -> dict:
        with self._lock:
            done = [r for r in self.completed if r.t_submit >= since and r.ok]
            waiting = len(self._pending)
        if not done:
            return {"completed": 0, "waiting": waiting}
        lat = np.array([r.latency for r in done])
        span = max(r.t_done for r in done) - min(r.t_submit for r in done)
        wait = np.array([r.t_admit - r.t_submit for r in done])
        build = np.array([r.t_launched - r.t_admit for r in done])
        run = np.array([r.t_done - r.t_launched for r in done])
        return {
            "completed": len(done),
            "waiting": waiting,
            "throughput_rps": len(done) / span if span > 0 else float("nan"),
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3),
            "batches": self.batches_launched,
            "peak_admitted_bytes": self.peak_bytes,
            "mean_queue_ms": float(wait.mean() * 1e3),
            "mean_build_launch_ms": float(build.mean() * 1e3),
            "mean_device_ms": float(run.mean() * 1e3),
        }
