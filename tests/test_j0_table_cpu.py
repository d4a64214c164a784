"""The Bessel-sum kernel's J0 table for arguments below 25 (csrc/kr_j0_table.h).

The committed header must equal what its generator produces, and its piecewise Taylor
polynomials must reproduce SciPy's j0 to within 5e-16 absolute on [0, 25).
"""

import importlib.util
import re
from pathlib import Path

import numpy as np
from scipy.special import j0

CSRC = Path(__file__).resolve().parent.parent / "seismicinversion_b200" / "csrc"


def _table():
    txt = (CSRC / "kr_j0_table.h").read_text()
    rows = re.findall(r"\{([^{}]+)\},", txt)
    return np.array([[float(v) for v in r.split(",")] for r in rows])


def test_table_matches_generator():
    spec = importlib.util.spec_from_file_location("gen_j0_table", CSRC / "gen_j0_table.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    T = _table()
    assert T.shape == (gen.N_INTERVALS, gen.DEGREE + 1)
    from decimal import Decimal

    for k in (0, 7, 24):
        ref = [float(v) for v in gen.coefficients(Decimal(k) + Decimal("0.5"))]
        assert np.array_equal(T[k], np.array(ref)), k


def test_table_accuracy_vs_scipy():
    T = _table()
    x = np.linspace(0.0, 25.0, 400001)[:-1]
    k = np.minimum(np.floor(x).astype(int), len(T) - 1)
    t = x - (k + 0.5)
    v = np.zeros_like(x)
    for n in range(T.shape[1] - 1, -1, -1):
        v = v * t + T[k, n]
    assert np.max(np.abs(v - j0(x))) < 5e-16


def _hankel_a(k):
    num, den = 1.0, 1.0
    for j in range(1, k + 1):
        num *= -float((2 * j - 1) ** 2)
        den *= 8.0 * j
    return num / den


def _j0_asym(x, nt):
    """The kernel's j0_asym_scaled times its amplitude: sqrt(1 / (pi x)) (P u + Q y v) with
    u = cos x + sin x, v = cos x - sin x, y = 1 / x and nt terms of P and Q."""
    y = 1.0 / x
    q = y * y
    P = np.full_like(x, (-1.0) ** (nt - 1) * _hankel_a(2 * (nt - 1)))
    Q = np.full_like(x, (-1.0) ** (nt - 1) * _hankel_a(2 * (nt - 1) + 1))
    for m in range(nt - 2, -1, -1):
        P = P * q + (-1.0) ** m * _hankel_a(2 * m)
        Q = Q * q + (-1.0) ** m * _hankel_a(2 * m + 1)
    c, s = np.cos(x), np.sin(x)
    return (P * (c + s) + Q * (y * (c - s))) / np.sqrt(np.pi * x)


def test_hankel_branch_accuracy_vs_scipy():
    """The fast path's expansion lengths (7 / 5 / 4 / 3 / 2 terms from x = 25 / 60 / 100 / 300 /
    3000, as in kr_gather.cu) reproduce SciPy's j0 to within 1e-15 absolute in each range."""
    src = (CSRC / "kr_gather.cu").read_text()
    assert ("x_first >= 3000.0 ? 2 : x_first >= 300.0 ? 3 : x_first >= 100.0 ? 4"
            in src.replace("\n", " ").replace("  ", " ").replace("  ", " "))
    for lo, hi, nt in ((25, 60, 7), (60, 100, 5), (100, 300, 4), (300, 3000, 3),
                       (3000, 20000, 2)):
        x = np.linspace(lo, hi, 200001)
        err = np.max(np.abs(_j0_asym(x, nt) - j0(x)))
        assert err < 1e-15, (lo, hi, nt, err)
