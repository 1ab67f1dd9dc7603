"""Host restatement of the device post-step hooks (frg_hooks.cu), used as
the reference those kernels are checked against and as the host side of the
methods that select them.

zhang_shu_limit_: the positivity-preserving scaling of Zhang & Shu
(J. Comput. Phys. 229 (2010) 8918-8934).  Per element, with the mean taken
with the quadrature weights w_i w_j |J| (so element integrals are kept):
the density at every solution point is pulled toward the mean until it is
>= eps_rho, then all components are pulled toward the mean by the largest
theta in [0, 1] that keeps the pressure >= eps_p at every point (the root
of rho(t) (p(t) - eps_p), a quadratic along mean + t (u_k - mean)).
Elements whose mean is not admissible are left unchanged.
"""
from __future__ import annotations

import numpy as np


def _root01(a, b, c):
    if abs(a) < 1e-300:
        return min(max(-c / b, 0.0), 1.0) if b != 0.0 else 0.0
    disc = max(b * b - 4.0 * a * c, 0.0)
    q = -0.5 * (b + np.copysign(np.sqrt(disc), b))
    r1 = q / a
    r2 = c / q if q != 0.0 else 2.0
    t = 1.0
    if 0.0 <= r1 <= 1.0:
        t = min(t, r1)
    if 0.0 <= r2 <= 1.0:
        t = min(t, r2)
    return t


def _limit_element(U, ww, g1, er, ep):
    """U: [npts, neq] of one element (modified in place); ww: [npts].
    Points at zero density give infinite or NaN pressure and are scaled like
    any other point below eps_p (as on the device)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        _limit(U, ww, g1, er, ep)


def _limit(U, ww, g1, er, ep):
    neq = U.shape[1]
    wsum = 0.0
    mean = np.zeros(neq)
    for k in range(U.shape[0]):
        wsum += ww[k]
        mean += ww[k] * U[k]
    mean = mean / wsum
    mom = mean[1:neq - 1]
    pbar = g1 * (mean[-1] - 0.5 * float(np.dot(mom, mom)) / mean[0])
    if not (mean[0] > er) or not (pbar > ep):
        return
    rmin = min(mean[0], float(np.min(U[:, 0])))
    if rmin < er:
        th = (mean[0] - er) / (mean[0] - rmin)
        U[:, 0] = mean[0] + th * (U[:, 0] - mean[0])
    theta = 1.0
    for k in range(U.shape[0]):
        m = U[k, 1:neq - 1]
        pk = g1 * (U[k, -1] - 0.5 * float(np.dot(m, m)) / U[k, 0])
        if pk >= ep:
            continue
        d = U[k] - mean
        dm = d[1:neq - 1]
        a = g1 * (d[-1] * d[0] - 0.5 * float(np.dot(dm, dm)))
        b = g1 * (mean[-1] * d[0] + mean[0] * d[-1] - float(np.dot(mom, dm))) - ep * d[0]
        c = mean[0] * (pbar - ep)
        theta = min(theta, _root01(a, b, c))
    if theta < 1.0:
        U[...] = mean + theta * (U - mean)


def zhang_shu_limit_(state, eq, eps_rho: float = 1e-13, eps_p: float = 1e-13):
    """Apply the limiter to state.u in place (1D [Np, Nel, 3] or 2D
    [Np, Np, Nel, 4], the reference layout)."""
    g1 = eq.gamma - 1.0
    w = np.asarray(state.ops.w, dtype=np.float64)
    u = state.u
    if state.dim == 1:
        J = state.mesh.J
        for e in range(u.shape[1]):
            U = np.array(u[:, e, :])
            _limit_element(U, w * J[e], g1, eps_rho, eps_p)
            u[:, e, :] = U
        return state
    m = state.mesh
    np_ = u.shape[0]
    if state.metrics is not None:
        absJ = np.abs(np.asarray(state.metrics["J"], dtype=np.float64))
    else:
        e = np.arange(m.n_elements)
        absJ = np.broadcast_to(np.abs(m.Jx[e % m.nx] * m.Jy[e // m.nx])[None, None, :], u.shape[:3])
    ww2 = w[:, None] * w[None, :]
    solid = getattr(m, "solid", None)
    for e in range(u.shape[2]):
        if solid is not None and solid[e]:
            continue
        # points ordered i fastest, as on the device
        U = np.array(u[:, :, e, :]).transpose(1, 0, 2).reshape(np_ * np_, -1)
        ww = (ww2 * absJ[:, :, e]).T.reshape(-1)
        _limit_element(U, ww, g1, eps_rho, eps_p)
        u[:, :, e, :] = U.reshape(np_, np_, -1).transpose(1, 0, 2)
    return state
