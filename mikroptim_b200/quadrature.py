"""Gauss-Legendre pupil quadrature (Forbes) on the host.

Restates the rule of ``include/mikroptim/pupil/quadrature.hpp:40-134``: radial nodes
u_i = rho_i^2 on [0, 1] with weights W_i (sum 1) from Gauss-Legendre of order N, azimuths
phi_j = (2j + 1) pi / (2M) (Half pupil), (2j + 1) pi / M (Full pupil) or phi = 0 (Axis,
M = 1), sample index k = i * M + j, sample weight W_i / M.

The reference ships a generated table for N <= 16 (pupil/gauss_legendre_table.hpp, made by
tools/gen_gauss_legendre_table.py with 60-digit Newton iterations, printed with 21 digits).
Here the nodes are computed the same way -- Newton on P_N with the three-term recurrence in
50-digit decimal arithmetic -- and rounded once to double, which also covers N up to 32
(the reference caps N at 16).
"""

from __future__ import annotations

from decimal import Decimal, getcontext
from functools import lru_cache
import math

import numpy as np

MAX_RINGS = 32

PUPIL_HALF = 0
PUPIL_FULL = 1
PUPIL_AXIS = 2


def _legendre(n: int, x: Decimal) -> tuple[Decimal, Decimal]:
    """P_n(x) and P_n'(x) by the recurrence (k+1) P_{k+1} = (2k+1) x P_k - k P_{k-1}."""
    p0, p1 = Decimal(1), x
    if n == 0:
        return p0, Decimal(0)
    for k in range(1, n):
        p0, p1 = p1, ((2 * k + 1) * x * p1 - k * p0) / (k + 1)
    dp = n * (x * p1 - p0) / (x * x - 1)
    return p1, dp


@lru_cache(maxsize=None)
def gauss_legendre_unit(n: int) -> tuple[tuple[float, ...], tuple[float, ...]]:
    """Nodes u_i (ascending) and weights W_i (sum 1) of order n on [0, 1], as doubles."""
    if not 1 <= n <= MAX_RINGS:
        raise ValueError(f"pupil quadrature: rings must be in [1, {MAX_RINGS}], got {n}")
    getcontext().prec = 50
    us, ws = [], []
    for i in range(n):
        # Chebyshev-like start for the i-th root of P_n on [-1, 1] (descending in i)
        x = Decimal(math.cos(math.pi * (i + 0.75) / (n + 0.5)))
        for _ in range(100):
            p, dp = _legendre(n, x)
            dx = p / dp
            x -= dx
            if abs(dx) < Decimal(10) ** -45:
                break
        _, dp = _legendre(n, x)
        w = 2 / ((1 - x * x) * dp * dp)
        us.append((1 + x) / 2)
        ws.append(w / 2)
    order = sorted(range(n), key=lambda i: us[i])
    return (tuple(float(us[i]) for i in order), tuple(float(ws[i]) for i in order))


def sample_count(rings: int, spokes: int, mode: int) -> int:
    """N * M samples per field (N for the Axis mode)."""
    return rings if mode == PUPIL_AXIS else rings * spokes


def samples(rings: int, spokes: int, mode: int) -> np.ndarray:
    """Samples (rho, phi, weight) of one field as an array [n, 3] (pupil/quadrature.hpp:71)."""
    u, w = gauss_legendre_unit(rings)
    m = 1 if mode == PUPIL_AXIS else spokes
    out = np.empty((rings * m, 3))
    pi = 3.14159265358979323846264338327950288
    for i in range(rings):
        for j in range(m):
            k = i * m + j
            out[k, 0] = math.sqrt(u[i])
            out[k, 2] = w[i] / float(m)
            if mode == PUPIL_HALF:
                out[k, 1] = float(2 * j + 1) * pi / float(2 * m)
            elif mode == PUPIL_FULL:
                out[k, 1] = float(2 * j + 1) * pi / float(m)
            else:
                out[k, 1] = 0.0
    return out
