"""Scoring metrics of the reference's 1D discontinuous cases, restated on the
host -- TEST INFRASTRUCTURE ONLY (the checker of the device-side
frg_shock_metrics_1d; the product package never imports this module).

Restates, with the reference's own evaluation order and Julia semantics
(NaN in max/min, isless for sorting, no fused multiply-add):

* sample_solution_1d       src/verification/Metrics.jl:95-123
* mean_sp_spacing          src/verification/Metrics.jl:126-130
* overshoot_metric         src/verification/Metrics.jl:81-87
* shock_thickness_sp       src/verification/Metrics.jl:138-200
* excess_dissipation       src/verification/Metrics.jl:208-223
* smooth_region_mask       src/verification/Metrics.jl:228-255
* interp_1d                src/verification/Metrics.jl:258-275
* sod_exact                src/verification/ExactSod.jl:20-163 (the exact
  Riemann solution of the Sod tube: Newton iteration for p*, star states,
  shock / rarefaction fans; Toro, Riemann Solvers and Numerical Methods for
  Fluid Dynamics, ch. 4)
"""
from __future__ import annotations

import bisect
import math

import numpy as np


def _jl_max(a: float, b: float) -> float:
    """Julia max on Float64: NaN wins."""
    if a != a:
        return a
    if b != b:
        return b
    return a if a >= b else b


def _jl_min(a: float, b: float) -> float:
    if a != a:
        return a
    if b != b:
        return b
    return a if a <= b else b


def _isless_key(v: float):
    """Sort key of Julia isless: -0.0 before 0.0, NaN last."""
    if v != v:
        return (2, 0.0, 0)
    return (0, v, 0 if math.copysign(1.0, v) < 0 else 1)


def sample_solution_1d(x_vertices, J, xi, u):
    """(x, rho) sorted by x from a 1D state u[j, e, c] (Metrics.jl:95-123);
    x = mid + J xi as Mesh1D.jl:45-52 evaluates it."""
    xv = np.asarray(x_vertices, dtype=np.float64)
    mid = (xv[:-1] + xv[1:]) / 2.0
    X = mid[None, :] + np.asarray(J, dtype=np.float64)[None, :] * np.asarray(xi, dtype=np.float64)[:, None]
    xs = X.T.ravel()  # idx = (e, j) with j fastest
    vs = np.asarray(u, dtype=np.float64)[:, :, 0].T.ravel()
    perm = np.argsort(xs, kind="stable")
    return xs[perm], vs[perm]


def mean_sp_spacing(x) -> float:
    n = len(x)
    if n < 2:
        return 1.0
    return (float(x[-1]) - float(x[0])) / (n - 1)


def overshoot_metric(u_min, u_max, u_ref_min, u_ref_max):
    D = _jl_max(abs(u_ref_max - u_ref_min), float(np.finfo(np.float64).eps))
    over = _jl_max(0.0, float(u_max) - float(u_ref_max)) / D
    under = _jl_max(0.0, float(u_ref_min) - float(u_min)) / D
    return over, under, _jl_max(over, under)


def steepest_gradient(x, rho):
    """0-based index of the first steepest |d rho| / max(|dx|, 1e-30)."""
    n = len(x)
    imax, gmax = 1, 0.0
    for i in range(1, n):
        g = abs(float(rho[i]) - float(rho[i - 1])) / max(abs(float(x[i]) - float(x[i - 1])), 1e-30)
        if g > gmax:
            gmax, imax = g, i
    return imax, gmax


def shock_thickness_sp(x, rho, window_sp: int = 30) -> float:
    """10%-90% rise distance of the steepest density jump in mean solution
    point spacings (Metrics.jl:138-200; plateaus from the window medians)."""
    n = len(x)
    if n < 4:
        return float("nan")
    imax0, _ = steepest_gradient(x, rho)
    r = [float(v) for v in rho]
    imax = imax0 + 1  # 1-based from here on, as the reference
    i0 = max(1, imax - window_sp)
    i1 = min(n, imax + window_sp)
    w = i1 - i0 + 1
    nL = max(1, w // 3)
    left = sorted(r[i0 - 1:i0 - 1 + nL], key=_isless_key)
    right = sorted(r[i1 - nL:i1], key=_isless_key)
    rL = left[max(1, len(left) // 2) - 1]
    rR = right[max(1, len(right) // 2) - 1]
    rmin, rmax = _jl_min(rL, rR), _jl_max(rL, rR)
    D = rmax - rmin
    if abs(D) < 1e-14:
        return float("nan")
    lo = rmin + 0.1 * D
    hi = rmin + 0.9 * D
    R = lambda i: r[i - 1]  # noqa: E731
    i10 = i90 = imax
    if rR >= rL:
        while i10 > i0 and R(i10) > lo:
            i10 -= 1
        while i90 < i1 and R(i90) < hi:
            i90 += 1
    else:
        while i10 < i1 and R(i10) > lo:
            i10 += 1
        while i90 > i0 and R(i90) < hi:
            i90 -= 1
    dx = abs(float(x[i90 - 1]) - float(x[i10 - 1]))
    return dx / mean_sp_spacing(x)


def smooth_region_mask(x, rho, grad_frac: float = 0.1, exclude_windows=()):
    n = len(x)
    g = [0.0] * n
    for i in range(1, n):
        g[i] = abs(float(rho[i]) - float(rho[i - 1])) / max(abs(float(x[i]) - float(x[i - 1])), 1e-30)
    g[0] = g[1]
    gmax = g[0]
    for v in g[1:]:
        gmax = _jl_max(gmax, v)
    thr = grad_frac * gmax
    mask = [True] * n
    for i in range(n):
        if g[i] > thr:
            mask[i] = False
        for a, b in exclude_windows:
            if a <= x[i] <= b:
                mask[i] = False
    return np.array(mask)


def excess_dissipation(u_method, u_ref, mask=None) -> float:
    num = den = 0.0
    for i in range(len(u_method)):
        if mask is not None and not mask[i]:
            continue
        num += abs(float(u_method[i]) - float(u_ref[i]))
        den += abs(float(u_ref[i]))
    return num / (den + 1e-30)


def l1_relative(rho, rho_ref) -> float:
    """sum(abs.(rho .- ref)) / (sum(abs.(ref)) + 1e-30) (Cases.jl:1021)."""
    return float(np.sum(np.abs(np.asarray(rho) - np.asarray(rho_ref))) / (np.sum(np.abs(rho_ref)) + 1e-30))


def interp_1d(x_ref, v_ref, xq):
    out = np.empty(len(xq))
    xr = [float(v) for v in x_ref]
    for i, xv in enumerate(xq):
        x = float(xv)
        if x <= xr[0]:
            out[i] = float(v_ref[0])
        elif x >= xr[-1]:
            out[i] = float(v_ref[-1])
        else:
            j = bisect.bisect_right(xr, x)  # searchsortedlast, 1-based
            j = min(max(j, 1), len(xr) - 1)
            t = (x - xr[j - 1]) / (xr[j] - xr[j - 1] + 1e-30)
            out[i] = (1 - t) * float(v_ref[j - 1]) + t * float(v_ref[j])
    return out


# ------------------------------------------------------------- exact Sod

def _sod_f_df(p, g, rL, pL, cL, rR, pR, cR, uL, uR):
    if p > pL:
        AL = 2.0 / ((g + 1) * rL)
        BL = (g - 1) / (g + 1) * pL
        ql = math.sqrt(AL / (p + BL))
        fL = (p - pL) * ql
        dfL = ql * (1.0 - 0.5 * (p - pL) / (p + BL))
    else:
        fL = 2 * cL / (g - 1) * ((p / pL) ** ((g - 1) / (2 * g)) - 1.0)
        dfL = (1 / (rL * cL)) * (p / pL) ** (-(g + 1) / (2 * g))
    if p > pR:
        AR = 2.0 / ((g + 1) * rR)
        BR = (g - 1) / (g + 1) * pR
        qr = math.sqrt(AR / (p + BR))
        fR = (p - pR) * qr
        dfR = qr * (1.0 - 0.5 * (p - pR) / (p + BR))
    else:
        fR = 2 * cR / (g - 1) * ((p / pR) ** ((g - 1) / (2 * g)) - 1.0)
        dfR = (1 / (rR * cR)) * (p / pR) ** (-(g + 1) / (2 * g))
    return fL + fR + (uR - uL), dfL + dfR


def sod_exact_density(x, t: float, gamma: float = 1.4, x0: float = 0.5):
    """Exact Sod density at the points x and time t (ExactSod.jl:103-163)."""
    g = gamma
    rL, uL, pL, rR, uR, pR = 1.0, 0.0, 1.0, 0.125, 0.0, 0.1
    cL, cR = math.sqrt(g * pL / rL), math.sqrt(g * pR / rR)
    p = max(0.5 * (pL + pR), 1e-8)
    tol = 1e-12
    for _ in range(60):
        f, df = _sod_f_df(p, g, rL, pL, cL, rR, pR, cR, uL, uR)
        if abs(f) < tol:
            break
        p = max(p - f / df, tol)
    ps = p
    if ps > pL:
        fL = (ps - pL) * math.sqrt((2.0 / ((g + 1) * rL)) / (ps + (g - 1) / (g + 1) * pL))
    else:
        fL = 2 * cL / (g - 1) * ((ps / pL) ** ((g - 1) / (2 * g)) - 1.0)
    if ps > pR:
        fR = (ps - pR) * math.sqrt((2.0 / ((g + 1) * rR)) / (ps + (g - 1) / (g + 1) * pR))
    else:
        fR = 2 * cR / (g - 1) * ((ps / pR) ** ((g - 1) / (2 * g)) - 1.0)
    us = 0.5 * (uL + uR) + 0.5 * (fR - fL)

    def rho_star(r, pp):
        if ps > pp:
            return r * (ps / pp + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pp + 1)
        return r * (ps / pp) ** (1 / g)

    rsL, rsR = rho_star(rL, pL), rho_star(rR, pR)
    out = np.empty(len(x))
    for i, xv in enumerate(x):
        xv = float(xv)
        if t <= 0.0:
            out[i] = rL if xv < x0 else rR
            continue
        xi = (xv - x0) / t
        if xi < us:
            if ps > pL:
                sL = uL - cL * math.sqrt((g + 1) / (2 * g) * ps / pL + (g - 1) / (2 * g))
                out[i] = rL if xi < sL else rsL
            else:
                sHL = uL - cL
                csL = cL * (ps / pL) ** ((g - 1) / (2 * g))
                sTL = us - csL
                if xi < sHL:
                    out[i] = rL
                elif xi < sTL:
                    c = (2 / (g + 1)) * (cL + ((g - 1) / 2) * (uL - xi))
                    out[i] = rL * (c / cL) ** (2 / (g - 1))
                else:
                    out[i] = rsL
            continue
        if ps > pR:
            sR = uR + cR * math.sqrt((g + 1) / (2 * g) * ps / pR + (g - 1) / (2 * g))
            out[i] = rR if xi > sR else rsR
        else:
            sHR = uR + cR
            csR = cR * (ps / pR) ** ((g - 1) / (2 * g))
            sTR = us + csR
            if xi > sHR:
                out[i] = rR
            elif xi > sTR:
                c = (2 / (g + 1)) * (cR - ((g - 1) / 2) * (uR - xi))
                out[i] = rR * (c / cR) ** (2 / (g - 1))
            else:
                out[i] = rsR
    return out
