"""Cubic B-spline EAM functions for the parameter-adjoint model.

The reference's EAM is analytic (eam.f90: Zhou terms; force.f90:256-351:
piecewise embedding), so the spline parameterisation is this library's: the
three functions of one metal M -- the density f_M(r) it contributes to any
neighbour, its pair potential with itself phi_MM(r) and its embedding
F_M(rho) -- each as a uniform cubic B-spline of 64 coefficients.  The
coefficients start as least-squares fits to the analytic forms, so the spline
model reproduces the analytic physics to the fit error.

Basis (the one the device evaluates): t = (x - x0) / h with h = (x1 - x0)/61,
interval i = floor(t) clamped to [0, 60], u = t - i,
s(x) = c[i] (1-u)^3/6 + c[i+1] (3u^3 - 6u^2 + 4)/6 + c[i+2] (-3u^3 + 3u^2 + 3u + 1)/6
       + c[i+3] u^3/6.
"""
from __future__ import annotations

import numpy as np

from ._abi import EamSpline, SPLINE_N


def basis_matrix(x: np.ndarray, x0: float, x1: float) -> np.ndarray:
    """Rows: the 64 basis values at each x (the device's clamped evaluation)."""
    h = (x1 - x0) / (SPLINE_N - 3)
    t = (np.asarray(x, dtype=np.float64) - x0) / h
    i = np.clip(np.floor(t).astype(np.int64), 0, SPLINE_N - 4)
    u = t - i
    v = 1.0 - u
    B = np.zeros((len(t), SPLINE_N))
    rows = np.arange(len(t))
    for m, b in enumerate((v ** 3 / 6.0, (3 * u ** 3 - 6 * u ** 2 + 4) / 6.0,
                           (-3 * u ** 3 + 3 * u ** 2 + 3 * u + 1) / 6.0, u ** 3 / 6.0)):
        B[rows, i + m] += b
    return B


def evaluate(c: np.ndarray, x: np.ndarray, x0: float, x1: float) -> np.ndarray:
    return basis_matrix(x, x0, x1) @ np.asarray(c)


def _zhou(r, A, re, c, lam):
    return A * np.exp(-c * (r / re - 1.0)) / (1.0 + (r / re - lam) ** 20)


def metal_functions(pot, metal: int = 1):
    """The analytic f_M(r), phi_MM(r) (eam.f90:3-35) and F_M(rho)
    (force.f90:256-315) of metal species `metal` (1 = Al) as numpy callables."""
    e = pot.eam[metal - 1]
    dens = lambda r: _zhou(r, e.f_e, e.r_e, e.beta, e.lambda_)
    phi = lambda r: _zhou(r, e.A, e.r_e, e.alpha, e.kappa) - _zhou(r, e.B, e.r_e, e.beta, e.lambda_)

    def emb(rho):
        rho = np.asarray(rho, dtype=np.float64)
        out = np.zeros_like(rho)
        rn, r0 = 0.85 * e.rho_e, 1.15 * e.rho_e
        for k, x in np.ndenumerate(rho):
            if x < rn:
                cf, rr = e.Fn, rn
            elif x < e.rho_e:
                cf, rr = e.Fm, e.rho_e
            elif x < r0:
                cf, rr = e.Fp, e.rho_e
            else:
                t = (x / e.rho_s) ** e.eta
                out[k] = e.Fe * (1.0 - np.log(t)) * t
                continue
            t = x / rr - 1.0
            out[k] = cf[0] + cf[1] * t + cf[2] * t * t + cf[3] * t ** 3
        return out

    return dens, phi, emb


def fit(pot, metal: int = 1, r0: float = 1.5, r1: float = 10.0, rho0: float = 0.0, rho1: float = 60.0,
        samples: int = 4000) -> EamSpline:
    """Least-squares spline fits of metal M's analytic EAM functions."""
    dens, phi, emb = metal_functions(pot, metal)
    s = EamSpline()
    s.metal, s.r0, s.r1, s.rho0, s.rho1 = metal, r0, r1, rho0, rho1
    r = np.linspace(r0, r1, samples)
    rho = np.linspace(rho0, rho1, samples)
    Br = basis_matrix(r, r0, r1)
    Bp = basis_matrix(rho, rho0, rho1)
    s.phi[:] = np.linalg.lstsq(Br, phi(r), rcond=None)[0]
    s.dens[:] = np.linalg.lstsq(Br, dens(r), rcond=None)[0]
    s.emb[:] = np.linalg.lstsq(Bp, emb(rho), rcond=None)[0]
    return s


def coefficients(s: EamSpline) -> np.ndarray:
    """The 192 spline coefficients in gradient order: phi, dens, emb."""
    return np.concatenate([np.array(s.phi), np.array(s.dens), np.array(s.emb)])


def with_coefficients(s: EamSpline, c: np.ndarray) -> EamSpline:
    t = EamSpline()
    t.metal, t.r0, t.r1, t.rho0, t.rho1 = s.metal, s.r0, s.r1, s.rho0, s.rho1
    t.phi[:] = c[:SPLINE_N]
    t.dens[:] = c[SPLINE_N:2 * SPLINE_N]
    t.emb[:] = c[2 * SPLINE_N:3 * SPLINE_N]
    return t
