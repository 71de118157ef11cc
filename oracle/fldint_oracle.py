"""CPU restatement of the reference's finite field integral.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of FldInt; the
product package never imports it.

The reference integrates each element's field along P1 -> P2 with the
composite Newton 3/8 rule (weights 3/8, 9/8, 9/8, 3/4, ..., 3/8 times the
step) on 3 * 2^k intervals, doubling k until the integral (times the segment
length) changes by less than PrcBInt in every component
(radTg3d::B_intCompFinNum, cpp/src/core/radg3d.cpp:258-342).  Because the
interval count stays a multiple of 3, reusing the old points with their old
weights (as the reference does) gives exactly the composite rule on the new
grid, which is what is evaluated here, on the total field of the geometry.
"""
from __future__ import annotations

import numpy as np


def newton38_weights(n_int: int) -> np.ndarray:
    """Composite Newton 3/8 weights for n_int intervals (a multiple of 3)."""
    w = np.empty(n_int + 1)
    k = np.arange(n_int + 1)
    w[:] = np.where(k % 3 == 0, 3.0 / 4.0, 9.0 / 8.0)
    w[0] = w[-1] = 3.0 / 8.0
    return w


def field_int_fin(field_fn, P1, P2, prec: float = 1e-3, max_doublings: int = 22):
    """Finite integral of field_fn (points [n, 3] -> values [n, 3]) from P1
    to P2 in T mm, following radg3d.cpp:258-342.  Returns (value, points)."""
    P1 = np.asarray(P1, dtype=float)
    P2 = np.asarray(P2, dtype=float)
    V = P2 - P1
    fact = float(np.linalg.norm(V))
    prev = np.full(3, 1e23)
    n_int = 3
    for _ in range(max_doublings):
        t = np.linspace(0.0, 1.0, n_int + 1)
        F = field_fn(P1[None, :] + t[:, None] * V[None, :])
        cur = (newton38_weights(n_int)[:, None] * F).sum(axis=0) / n_int
        if fact * np.abs(cur - prev).max() < prec:
            return fact * cur, n_int + 1
        prev = cur
        n_int *= 2
    raise RuntimeError("Newton 3/8 integral did not reach the requested precision")
