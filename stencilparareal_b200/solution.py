"""Analytic solution and error measures of the advection-diffusion problem.

Restates src/Convection/ConvectionSolution.h of the reference: exactQ (:8-20),
fillQ on the unit cube (:23-52), computeError (:55-103); and
computeErrorReference of src/Parareal/main.cpp:98-139.  Vectorised with numpy
over dense (nk, nj, ni) arrays (i fastest); x = (i+1/2)/ni pairs with i.
"""
from __future__ import annotations

import numpy as np

PI = 3.14159265358979  # the reference's value (ConvectionSolution.h:11)


def exact_q(nu0: float, nufreq: float, cx: float, cy: float, cz: float, x, y, z, t: float):
    """exactQ: sin2pi(x-cx t) sin2pi(y-cy t) sin2pi(z-cz t) exp(-12 pi^2 a(t))."""
    a = nu0 * t - (nu0 / (2.0 * nufreq)) * (np.cos(nufreq * t) - 1.0) if nufreq > 0 else nu0 * t
    return (np.sin(2.0 * PI * (x - cx * t)) * np.sin(2.0 * PI * (y - cy * t)) * np.sin(2.0 * PI * (z - cz * t))
            * np.exp(-12.0 * PI * PI * a))


def fill_q(ni: int, nj: int, nk: int, nu0: float, nufreq: float, cx: float, cy: float, cz: float, t: float):
    """fillQ on [0,1]^3 at time t: the field at the cell centres, shape (nk, nj, ni)."""
    x = (2 * np.arange(ni) + 1) * (1.0 / ni / 2.0)
    y = (2 * np.arange(nj) + 1) * (1.0 / nj / 2.0)
    z = (2 * np.arange(nk) + 1) * (1.0 / nk / 2.0)
    zz, yy, xx = np.meshgrid(z, y, x, indexing="ij")
    return exact_q(nu0, nufreq, cx, cy, cz, xx, yy, zz, t)


def compute_error(q, nu0, nufreq, cx, cy, cz, t):
    """computeError: (max|q - exact|, max|exact|, their ratio) at time t."""
    nk, nj, ni = q.shape
    ex = fill_q(ni, nj, nk, nu0, nufreq, cx, cy, cz, t)
    e_inf = float(np.abs(q - ex).max())
    x_inf = float(np.abs(ex).max())
    return e_inf, x_inf, e_inf / x_inf


def error_reference(field, reference) -> float:
    """computeErrorReference: max|field - reference| / max|field|."""
    return float(np.abs(field - reference).max() / np.abs(field).max())
