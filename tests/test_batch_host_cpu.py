"""Host logic of the batch launcher that needs no GPU: the allocation size classes of a batch's
single device block (four classes per power of two, at least 1 MiB)."""

import numpy as np

from seismicinversion_b200.batch import SCHEDULES, _size_class


def test_size_classes():
    rng = np.random.default_rng(0)
    sizes = np.r_[0, 1, 1 << 20, (1 << 20) + 1, 3 << 20, rng.integers(1, 1 << 34, 2000)]
    classes = set()
    for n in sizes:
        c = _size_class(int(n))
        assert c >= max(int(n), 1 << 20)
        assert c <= max(int(n), 1 << 20) * 1.25  # at most 25 % slack
        assert _size_class(c) == c  # a class is its own class
        classes.add(c)
    # four classes per power of two: 1.25, 1.5, 1.75 and 2 times the power below
    per_octave = [sum(1 for c in classes if (1 << k) < c <= (1 << (k + 1))) for k in range(20, 34)]
    assert max(per_octave) <= 4


def test_schedules_are_valid_configurations():
    for threads, tile_w in SCHEDULES:
        assert threads in (32, 64, 128) and 32 <= tile_w <= 8192


def test_request_bytes_bounds_the_batch_footprint():
    """serve.request_bytes is an upper bound on a request's device footprint: its buffers and
    its plan (kr_batch_plan_bytes, host-only, for the server's schedule) times the 1.25 slack of
    the batch block's size class, for random model depths, grids and request kinds."""
    import ctypes

    from seismicinversion_b200 import _lib
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.serve import request_bytes

    h = _lib.lib()
    cfg = _lib.BatchConfig(128, 256, 0, 0)  # GpuBatchExecutor's schedule
    rng = np.random.default_rng(0)
    for t in range(200):
        n_sub = int(rng.integers(2, 64))
        n_p = int(rng.integers(1, 257))
        n_w = int(rng.choice([16, 256, 512, 1024, 2048]))
        grad = bool(rng.random() < 0.5)
        m = random_layered_model(n_sub, seed=t)
        L = m.n_layers
        desc = np.zeros(1, dtype=_lib.MODEL_DESC_FIELDS)
        desc["n_layers"], desc["n_p"], desc["n_w"] = L, n_p, n_w
        desc["flags"] = (_lib.KR_BATCH_GRADIENT | _lib.KR_BATCH_STORE_R) if grad else 0
        plan = h.kr_batch_plan_bytes(desc.ctypes.data, 1, ctypes.byref(cfg))
        assert plan > 0
        buf = 48 * L + 8 * n_p + 16 * n_w + 16 * n_p * n_w
        if grad:
            buf += 16 * n_p * n_w + 8 * (4 * L + 1)
        assert request_bytes(m, n_p, n_w, grad) >= 1.25 * (buf + plan), (L, n_p, n_w, grad)


class _FakeBatch:
    """Stands in for a ModelBatch: a signature and a schedule setter; launch time per schedule
    comes from a table (the timing itself is patched)."""

    def __init__(self, sig, costs):
        self.sig, self.costs, self.schedule, self.set_calls = sig, costs, None, 0

    def signature(self):
        return self.sig

    def set_schedule(self, sch):
        self.schedule = tuple(sch)
        self.set_calls += 1


def test_autotune_picks_fastest_and_caches(tmp_path, monkeypatch):
    import json

    from seismicinversion_b200 import batch as B

    monkeypatch.setattr(B, "_time_launch", lambda b, reps: b.costs[b.schedule])
    monkeypatch.setattr(B, "_TUNE_CACHE", {})
    costs = {(32, 128): 5.0, (128, 256): 2.0, (128, 512): 1.5, (64, 128): 3.0}
    cache = tmp_path / "tune.json"
    fb = _FakeBatch("sigA", costs)
    best, times = B.autotune(fb, candidates=list(costs), cache_file=str(cache))
    assert best == (128, 512) and fb.schedule == (128, 512) and times == costs
    assert json.loads(cache.read_text()) == {"sigA": [128, 512]}
    # memory cache: no timing on the second call
    fb2 = _FakeBatch("sigA", {})
    assert B.autotune(fb2, candidates=list(costs)) == ((128, 512), {})
    assert fb2.schedule == (128, 512) and fb2.set_calls == 1
    # disk cache survives a fresh process (empty memory cache)
    monkeypatch.setattr(B, "_TUNE_CACHE", {})
    fb3 = _FakeBatch("sigA", {})
    assert B.autotune(fb3, cache_file=str(cache))[0] == (128, 512)
    # a corrupt cache file is ignored and rewritten
    cache.write_text("{not json")
    fb4 = _FakeBatch("sigB", costs)
    assert B.autotune(fb4, candidates=list(costs), cache_file=str(cache))[0] == (128, 512)
    assert json.loads(cache.read_text()) == {"sigB": [128, 512]}
