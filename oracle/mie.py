"""Monostatic RCS of a perfectly conducting sphere (Mie series), the analytic
oracle of the reference's validation (util/monostatic_PEC_sphere.py:8-58).

Test infrastructure only.  Restated from the standard series

    sigma / (pi r^2) = (4 / x^2) | sum_{n>=1} (-1)^n (n + 1/2) (a_n - b_n) |^2,
    a_n = -[x j_n(x)]' / [x h_n(x)]',   b_n = -j_n(x) / h_n(x),   x = k r,

with h_n = j_n + i y_n (spherical Hankel, first kind) and the series truncated at
N = floor(x + 4 x^(1/3) + 2) terms.  Like the reference function it returns 0
for x <= 0 and 1 (the optical limit) for x >= 1000.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import spherical_jn, spherical_yn

C0 = 299792458.0


def normalized_rcs(x: float) -> float:
    """sigma / (pi r^2) at size parameter x = 2 pi r / lambda."""
    if x <= 0:
        return 0.0
    if x >= 1e3:
        return 1.0
    nmax = int(math.floor(x + 4.0 * x ** (1.0 / 3.0) + 2.0))
    n = np.arange(1, nmax + 1)
    j = spherical_jn(n, x)
    jd = spherical_jn(n, x, derivative=True)
    y = spherical_yn(n, x)
    yd = spherical_yn(n, x, derivative=True)
    h = j + 1j * y
    hd = jd + 1j * yd
    a = -(j + x * jd) / (h + x * hd)
    b = -j / h
    s = np.sum(((-1.0) ** n) * (n + 0.5) * (a - b))
    return float((4.0 / x ** 2) * abs(s) ** 2)


def sphere_rcs(radius_m: float, freq_hz: float) -> float:
    """Monostatic sigma (m^2) of a PEC sphere."""
    x = 2.0 * math.pi * radius_m * freq_hz / C0
    return normalized_rcs(x) * math.pi * radius_m ** 2
