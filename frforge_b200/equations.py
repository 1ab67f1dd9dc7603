"""Compressible Euler equations, host side (src/equations/Euler.jl, Euler2D.jl).

Used for initial conditions and host diagnostics; the residual itself runs in
the CUDA library.
"""
from __future__ import annotations

import numpy as np

EPS = np.finfo(np.float64).eps


class Euler1D:
    """1D Euler, conserved (rho, rho u, E), ideal gas (Euler.jl:9-16)."""

    neq = 3

    def __init__(self, gamma: float = 1.4):
        self.gamma = float(gamma)

    def primitives_to_conserved(self, rho, u, p):
        rho, u, p = (np.asarray(v, dtype=np.float64) for v in (rho, u, p))
        E = p / (self.gamma - 1.0) + 0.5 * rho * u * u
        return np.stack(np.broadcast_arrays(rho, rho * u, E), axis=-1)

    def pressure(self, U):
        U = np.asarray(U)
        rs = np.maximum(U[..., 0], EPS)
        u = U[..., 1] / rs
        return (self.gamma - 1.0) * (U[..., 2] - 0.5 * rs * u * u)

    def velocity(self, U):
        U = np.asarray(U)
        return U[..., 1] / np.maximum(U[..., 0], EPS)


class Euler2D:
    """2D Euler, conserved (rho, rho u, rho v, E) (Euler2D.jl:8-25)."""

    neq = 4

    def __init__(self, gamma: float = 1.4):
        self.gamma = float(gamma)

    def primitives_to_conserved(self, rho, u, v, p):
        rho, u, v, p = (np.asarray(x, dtype=np.float64) for x in (rho, u, v, p))
        E = p / (self.gamma - 1.0) + 0.5 * rho * (u * u + v * v)
        return np.stack(np.broadcast_arrays(rho, rho * u, rho * v, E), axis=-1)

    def pressure(self, U):
        U = np.asarray(U)
        r = np.maximum(U[..., 0], EPS)
        u = U[..., 1] / r
        v = U[..., 2] / r
        return (self.gamma - 1.0) * (U[..., 3] - 0.5 * r * (u * u + v * v))
