"""Host logic of the continuous-batching server with a fake executor (no GPU):
admission by memory budget (held results stay charged until released), FIFO order, rejection
of requests that can never fit, queue-full and invalid requests, cancellation of waiting
requests, bounded in-flight batches."""

import threading
import time

import numpy as np
import pytest

from seismicinversion_b200.earth_models import random_layered_model
from seismicinversion_b200.serve import KennettServer, RequestRejected, request_bytes


class FakeExecutor:
    """Completes each launched group after `delay` seconds; records what it saw."""

    def __init__(self, delay=0.02):
        self.delay = delay
        self.groups = []
        self.max_concurrent = 0
        self._live = 0
        self._lock = threading.Lock()

    def launch(self, reqs):
        with self._lock:
            self.groups.append([r.id for r in reqs])
            self._live += 1
            self.max_concurrent = max(self.max_concurrent, self._live)
        return {"t": time.perf_counter() + self.delay, "n": len(reqs)}

    def ready(self, h):
        if time.perf_counter() >= h["t"]:
            with self._lock:
                if not h.get("counted"):
                    h["counted"] = True
                    self._live -= 1
            return True
        return False

    def results(self, h, reqs):
        return [{"R": len(r.p) * len(r.omega)} for r in reqs]


def _req(srv, n_p=4, n_w=16, grad=False, seed=0):
    m = random_layered_model(3, seed=seed)
    p = np.linspace(0.1, 0.5, n_p)
    w = np.arange(1, n_w + 1) * 0.1
    obs = np.zeros((n_p, n_w), complex) if grad else None
    return srv.submit(m, p, w, gradient=grad, R_obs=obs)


def test_all_complete_fifo_and_inflight_bound():
    ex = FakeExecutor(delay=0.01)
    with KennettServer(executor=ex, max_batch_requests=4, max_inflight=2) as srv:
        reqs = [_req(srv, seed=i) for i in range(40)]
        for r in reqs:
            r.wait(10)
    flat = [i for g in ex.groups for i in g]
    assert flat == sorted(flat) == list(range(40))  # FIFO admission
    assert all(len(g) <= 4 for g in ex.groups)
    assert ex.max_concurrent <= 2
    st = srv.stats()
    assert st["completed"] == 40 and st["p99_ms"] >= st["p50_ms"] > 0


def test_budget_admission_waits_and_never_exceeds():
    m = random_layered_model(3, seed=0)
    one = request_bytes(m, 4, 16, False)
    ex = FakeExecutor(delay=0.02)
    with KennettServer(executor=ex, hbm_budget_bytes=3 * one, max_batch_requests=100,
                       max_inflight=4) as srv:
        reqs = [_req(srv) for _ in range(12)]
        for r in reqs:
            r.wait(10)
            r.release()  # the client consumes each result: its bytes return to the budget
        assert srv.peak_bytes <= 3 * one
    assert all(len(g) <= 3 for g in ex.groups) and len(ex.groups) >= 4


def test_rejections():
    ex = FakeExecutor()
    m = random_layered_model(3, seed=0)
    with KennettServer(executor=ex, hbm_budget_bytes=request_bytes(m, 4, 16, False)) as srv:
        big = _req(srv, n_p=64, n_w=512)
        with pytest.raises(RequestRejected, match="budget"):
            big.wait(1)
        bad = srv.submit(m, [0.1], [1.0], gradient=True)  # no R_obs
        with pytest.raises(RequestRejected):
            bad.wait(1)
        from seismicinversion_b200.layer_model import LayerModel

        elastic_top = LayerModel(m.alpha, np.r_[0.5, m.beta[1:]], m.rho, m.thickness, m.Q_alpha,
                                 m.Q_beta)
        with pytest.raises(RequestRejected):
            srv.submit(elastic_top, [0.1], [1.0]).wait(1)
        with pytest.raises(RequestRejected):
            srv.submit(m, [], [1.0]).wait(1)
    with KennettServer(executor=FakeExecutor(delay=0.5), max_pending=2, max_inflight=1,
                       max_batch_requests=1) as srv:
        rs = [_req(srv) for _ in range(6)]
        rejected = [r for r in rs if r.done.is_set() and r.error is not None]
        assert rejected and all("queue full" in str(r.error) for r in rejected)


def test_cancel_waiting_request():
    ex = FakeExecutor(delay=0.2)
    with KennettServer(executor=ex, max_batch_requests=1, max_inflight=1) as srv:
        first = _req(srv)
        time.sleep(0.02)
        second = _req(srv)
        assert srv.cancel(second)
        with pytest.raises(RequestRejected, match="cancelled"):
            second.wait(1)
        first.wait(5)
        assert not srv.cancel(first)
    assert [second.id] not in ex.groups


def test_held_results_hold_budget():
    """A completed request's bytes stay charged while its results are held (the results are
    views of its batch's device block); release() or dropping them returns the bytes."""
    m = random_layered_model(3, seed=0)
    one = request_bytes(m, 4, 16, False)
    ex = FakeExecutor(delay=0.005)
    with KennettServer(executor=ex, hbm_budget_bytes=2 * one, max_batch_requests=1,
                       max_inflight=2) as srv:
        a, b = _req(srv), _req(srv)
        a.wait(5)
        b.wait(5)
        assert srv.used_bytes == 2 * one
        c = _req(srv)
        time.sleep(0.2)
        assert not c.done.is_set()  # waits: a and b still hold their results
        held = a.result  # a result dict on its own keeps a's batch charged
        a.release()
        time.sleep(0.2)
        assert not c.done.is_set() and srv.used_bytes == 2 * one
        del held
        c.wait(5)  # a's bytes came back: c was admitted
        b.release()
        c.release()
    assert srv.used_bytes == 0


def test_server_leaves_global_gc_state_alone():
    import gc

    before = gc.get_freeze_count()
    with KennettServer(executor=FakeExecutor()) as srv:
        _req(srv).wait(5)
    assert gc.get_freeze_count() == before
