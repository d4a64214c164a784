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
