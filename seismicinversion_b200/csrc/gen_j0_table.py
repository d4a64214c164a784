"""Generate ``kr_j0_table.h``: piecewise Taylor coefficients of J0 on [0, 25).

Run from this folder (``python gen_j0_table.py``); the header is committed.

Interval k (k = 0..24) covers [k, k + 1) and is expanded about its centre c = k + 1/2:

    J0(c + t) = sum_{n=0}^{15} a_n t^n,   |t| <= 1/2.

a_0 = J0(c) and a_1 = -J1(c) come from the power series
J0(x) = sum_m (-1)^m (x/2)^(2m) / (m!)^2 and J1(x) = sum_m (-1)^m (x/2)^(2m+1) / (m! (m+1)!)
in 60-digit decimal arithmetic (the series cancels heavily for x ~ 25, hence the precision).
The remaining coefficients follow from Bessel's equation x y'' + y' + x y = 0 written about c:

    c (n+2)(n+1) a_{n+2} = -[(n+1)^2 a_{n+1} + c a_n + a_{n-1}],   a_{-1} = 0.

Since |J0^(n)| <= 1, the truncation error after degree 15 is below 0.5^16 / 16! < 1e-18.
"""

from __future__ import annotations

from decimal import Decimal, getcontext
from pathlib import Path

getcontext().prec = 60

N_INTERVALS = 25
DEGREE = 15


def _series(x: Decimal, order: int) -> Decimal:
    half = x / 2
    term = half**order
    for k in range(1, order + 1):
        term /= k
    total = Decimal(0)
    m = 0
    while True:
        total += term
        m += 1
        term = -term * half * half / (m * (m + order))
        if abs(term) < Decimal(10) ** -55 and m > 5:
            return total


def coefficients(c: Decimal) -> list[Decimal]:
    a = [_series(c, 0), -_series(c, 1)]
    prev = Decimal(0)  # a_{n-1}
    for n in range(0, DEGREE - 1):
        nxt = -((n + 1) ** 2 * a[n + 1] + c * a[n] + (a[n - 1] if n >= 1 else prev))
        a.append(nxt / (c * (n + 2) * (n + 1)))
    return a


def main() -> None:
    rows = []
    for k in range(N_INTERVALS):
        c = Decimal(k) + Decimal("0.5")
        rows.append([float(v) for v in coefficients(c)])
    lines = [
        "// Generated by gen_j0_table.py: J0(k + 1/2 + t) = sum_n kJ0Taylor[k][n] t^n, |t| <= 1/2.",
        "#pragma once",
        "",
        "namespace kr {",
        "",
        f"constexpr int kJ0TabIntervals = {N_INTERVALS};",
        f"constexpr int kJ0TabDegree = {DEGREE};",
        "",
        f"__device__ const double kJ0Taylor[{N_INTERVALS}][{DEGREE + 1}] = {{",
    ]
    for row in rows:
        lines.append("    {" + ", ".join(repr(v) for v in row) + "},")
    lines += ["};", "", "}  // namespace kr", ""]
    Path(__file__).with_name("kr_j0_table.h").write_text("\n".join(lines))


if __name__ == "__main__":
    main()
