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
