"""CPU restatement of the reference's electron trajectory integrator.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of FldPtcTrj;
the product package never imports it.

State F = (x, dx/dy, z, dz/dy) along the longitudinal coordinate y, with
dF/dy from the Lorentz force of the source field at (x, y, z)
(radTPrtclTrj::TrjEqs, cpp/src/core/radptrj.h:91-105).  Tabulation at np
equidistant points: one classical fourth-order Runge-Kutta step per interval
(radptrj.cpp:94-147), or, when accuracies are given, the step-doubling
control of RungeKuttaStep5 / AutoPropagate (radptrj.cpp:149-240).  field_fn
maps one point [3] to B [3].
"""
from __future__ import annotations

import math

import numpy as np


def _eqs(field_fn, ctm, s, F):
    xd, zd = F[1], F[3]
    buf = ctm * math.sqrt(1.0 + xd * xd + zd * zd)
    B = field_fn(np.array([F[0], s, F[2]]))
    return np.array([xd, -buf * (zd * B[1] - (1.0 + xd * xd) * B[2] + xd * zd * B[0]),
                     zd, buf * (xd * B[1] - (1.0 + zd * zd) * B[0] + xd * zd * B[2])])


def _rk4(field_fn, ctm, y, dydx, x, h):
    hh = 0.5 * h
    k2 = _eqs(field_fn, ctm, x + hh, y + hh * dydx)
    k3 = _eqs(field_fn, ctm, x + hh, y + hh * k2)
    k4 = _eqs(field_fn, ctm, x + h, y + h * k3)
    return y + (h / 6.0) * (dydx + k4 + 2.0 * (k2 + k3))


def _step5(field_fn, ctm, y, x, htry, prec, eps_tol=1.0):
    dydx = _eqs(field_fn, ctm, x, y)
    h = htry
    for _ in range(200):
        hh = 0.5 * h
        ymid = _rk4(field_fn, ctm, y, dydx, x, hh)
        y2 = _rk4(field_fn, ctm, ymid, _eqs(field_fn, ctm, x + hh, ymid), x + hh, hh)
        if x + h == x:
            raise RuntimeError("Radia::Error200")
        y1 = _rk4(field_fn, ctm, y, dydx, x, h)
        d = y2 - y1
        errmax = float(np.max(np.abs(d / prec))) / eps_tol
        if errmax <= 1.0:
            hnext = 0.9 * h * math.exp(-0.2 * math.log(errmax)) if errmax > 6.0e-04 else 4.0 * h
            return y2 + d / 15.0, x + h, h, hnext
        h *= 0.9 * math.exp(-0.25 * math.log(errmax))
    raise RuntimeError("no acceptable step")


def _propagate(field_fn, ctm, y, x1, x2, h1, hmin, prec, max_steps=5000):
    x, h = x1, (abs(h1) if x2 > x1 else -abs(h1))
    for _ in range(max_steps):
        if (x + h - x2) * (x + h - x1) > 0.0:
            h = x2 - x
        y, x, _, hnext = _step5(field_fn, ctm, y, x, h, prec)
        if (x - x2) * (x2 - x1) >= 0.0:
            return y
        if abs(hnext) <= hmin:
            raise RuntimeError("Radia::Error200")
        h = hnext
    raise RuntimeError("Radia::Error201")


def trajectory(field_fn, energy_gev, init, y0, y1, np_, prec=None):
    """[np_, 5] rows (y, x, dx/dy, z, dz/dy) from init (x, x', z, z') at y0."""
    ctm = -2.99792458e+05 / (1.e+09 * energy_gev)
    step = (y1 - y0) / (np_ - 1) if np_ > 1 else 0.0
    pr = None if prec is None else np.array([1e23 if p == 0.0 else p for p in prec], dtype=float)
    Y = np.array(init, dtype=float)
    x = float(y0)
    out = np.zeros((np_, 5))
    for i in range(np_):
        out[i, 0] = x
        out[i, 1:] = Y
        if i == np_ - 1:
            break
        x1 = x + step
        if pr is None:
            Y = _rk4(field_fn, ctm, Y, _eqs(field_fn, ctm, x, Y), x, step)
        else:
            Y = _propagate(field_fn, ctm, Y, x, x1, step, 1e-10 * step, pr)
        x = x1
    return out
