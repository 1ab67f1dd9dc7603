"""Meshes and boundary conditions (src/mesh/Mesh1D.jl, Mesh2D.jl,
BoundaryConditions.jl, MeshMetrics2D.jl).

Element vertices follow the reference's ``collect(range(a, b; length))``
(exact rational progression, each element rounded once) so element sizes
match the reference bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from fractions import Fraction
from typing import Optional, Sequence

import numpy as np

from .operators import FROperators


class AbstractBC:
    kind = "abstract"


class PeriodicBC(AbstractBC):
    kind = "periodic"


class TransmissiveBC(AbstractBC):
    """Zero-order extrapolation: ghost = interior trace."""

    kind = "transmissive"


class ReflectingBC(AbstractBC):
    """Slip wall: reverse the normal velocity (reflect_conserved)."""

    kind = "reflecting"


@dataclass
class DirichletBC(AbstractBC):
    """Prescribed conserved state.  The GPU path takes a constant state; a
    time- or space-dependent ``u_func`` has no device form and is rejected."""

    state: Sequence[float]
    kind: str = field(default="dirichlet", init=False)


@dataclass
class XSplitGhostBC(AbstractBC):
    """GhostStateBC of the double-Mach case (Cases2D_Optional.jl:72-84):
    ghost = ``state`` for x < x0 + (s0 + s1*t)/sdiv, otherwise the reflected
    interior state (``right_reflect``) or ``state_b``."""

    state: Sequence[float]
    x0: float
    s0: float = 0.0
    s1: float = 0.0
    sdiv: float = 1.0
    right_reflect: bool = True
    state_b: Optional[Sequence[float]] = None
    kind: str = field(default="xsplit", init=False)


def is_periodic(bc: AbstractBC) -> bool:
    return isinstance(bc, PeriodicBC)


def _rat(x: float):
    """Base.rat: continued-fraction numerator/denominator (limit 2^24)."""
    y = x
    a, d, b, c = 1, 1, 0, 0
    m = 16777216.0
    while abs(y) <= m:
        f = int(np.trunc(y))
        y -= f
        a, c = f * a + c, a
        b, d = f * b + d, b
        if not (abs(a) <= m and abs(b) <= m):
            return c, d
        if a / b == x:
            break
        y = 1.0 / y
    return a, b


def julia_range(a: float, b: float, length: int) -> np.ndarray:
    """collect(range(a, b; length)) for Float64 endpoints."""
    if length == 1:
        return np.array([a], dtype=np.float64)
    an, ad = _rat(a)
    bn, bd = _rat(b)
    if ad != 0 and bd != 0:
        den = ad * bd // np.gcd(ad, bd)
        sn, en = round(den * a), round(den * b)
        if sn / den == a and en / den == b:
            return np.array([float(Fraction((length - i) * sn + (i - 1) * en, (length - 1) * den))
                             for i in range(1, length + 1)])
    return np.array([a + (b - a) * (i - 1) / (length - 1) for i in range(1, length + 1)])


class Mesh1D:
    """Uniform 1D mesh (Mesh1D.jl:23-42): vertices, dx, J = dx/2, end BCs."""

    def __init__(self, x_left, x_right, n_elements, left_bc=None, right_bc=None):
        left_bc = left_bc or PeriodicBC()
        right_bc = right_bc or PeriodicBC()
        if n_elements < 1:
            raise ValueError("n_elements must be >= 1")
        if not x_right > x_left:
            raise ValueError("x_right must be > x_left")
        if is_periodic(left_bc) != is_periodic(right_bc):
            raise ValueError("Periodic BC must be set on both ends")
        self.n_elements = int(n_elements)
        self.x_left, self.x_right = float(x_left), float(x_right)
        self.x_vertices = julia_range(float(x_left), float(x_right), n_elements + 1)
        self.dx = np.diff(self.x_vertices)
        self.J = self.dx / 2.0
        self.left_bc, self.right_bc = left_bc, right_bc

    def physical_coords(self, ops: FROperators) -> np.ndarray:
        """SP coordinates [Np, Nel] (Mesh1D.jl:45-63)."""
        mid = (self.x_vertices[:-1] + self.x_vertices[1:]) / 2.0
        return mid[None, :] + self.J[None, :] * ops.xi[:, None]


class Mesh2D:
    """Structured nx x ny quad mesh, e = (jy-1)*nx + jx (Mesh2D.jl:11-154)."""

    def __init__(self, x_left, x_right, y_bottom, y_top, nx, ny, left_bc=None, right_bc=None,
                 bottom_bc=None, top_bc=None, solid=None):
        left_bc = left_bc or PeriodicBC()
        right_bc = right_bc or PeriodicBC()
        bottom_bc = bottom_bc or PeriodicBC()
        top_bc = top_bc or PeriodicBC()
        if nx < 1 or ny < 1:
            raise ValueError("nx, ny must be >= 1")
        if not x_right > x_left:
            raise ValueError("x_right > x_left required")
        if not y_top > y_bottom:
            raise ValueError("y_top > y_bottom required")
        if is_periodic(left_bc) != is_periodic(right_bc):
            raise ValueError("x-periodic requires both left and right PeriodicBC")
        if is_periodic(bottom_bc) != is_periodic(top_bc):
            raise ValueError("y-periodic requires both bottom and top PeriodicBC")
        self.nx, self.ny = int(nx), int(ny)
        self.n_elements = self.nx * self.ny
        self.x_left, self.x_right, self.y_bottom, self.y_top = map(float, (x_left, x_right, y_bottom, y_top))
        self.x_vertices = julia_range(self.x_left, self.x_right, nx + 1)
        self.y_vertices = julia_range(self.y_bottom, self.y_top, ny + 1)
        self.dx = np.diff(self.x_vertices)
        self.dy = np.diff(self.y_vertices)
        self.Jx = self.dx / 2.0
        self.Jy = self.dy / 2.0
        self.left_bc, self.right_bc, self.bottom_bc, self.top_bc = left_bc, right_bc, bottom_bc, top_bc
        if solid is not None:
            solid = np.asarray(solid, dtype=bool).ravel()
            if solid.size != self.n_elements:
                raise ValueError(f"solid mask length must be n_elements={self.n_elements}")
        self.solid = solid
        self.wavy_amp: Optional[float] = None

    def element_index(self, jx: int, jy: int) -> int:
        """1-based (jx, jy) -> 1-based e (Mesh2D.jl:162-163)."""
        return (jy - 1) * self.nx + jx

    def element_coords(self, e: int):
        jy, r = divmod(e - 1, self.nx)
        return r + 1, jy + 1

    def physical_coords(self, ops: FROperators):
        """SP coordinates X, Y [Np, Np, Nel] (physical_xy, MeshMetrics2D.jl:49-74)."""
        xc = (self.x_vertices[:-1] + self.x_vertices[1:]) / 2.0
        yc = (self.y_vertices[:-1] + self.y_vertices[1:]) / 2.0
        e = np.arange(self.n_elements)
        jx, jy = e % self.nx, e // self.nx
        X = xc[jx][None, None, :] + self.Jx[jx][None, None, :] * ops.xi[:, None, None]
        Y = yc[jy][None, None, :] + self.Jy[jy][None, None, :] * ops.xi[None, :, None]
        X, Y = np.broadcast_arrays(X, Y)
        if self.wavy_amp is not None:
            a = self.wavy_amp
            x = X + a * np.sin(2 * np.pi * Y) * np.sin(np.pi * X)
            y = Y + a * np.sin(2 * np.pi * X) * np.sin(np.pi * Y)
            return x, y
        return X.copy(), Y.copy()


def make_wavy_mesh2d(nx, ny, ops=None, amp=0.05, x_left=0.0, x_right=1.0, y_bottom=0.0, y_top=1.0,
                     left_bc=None, right_bc=None, bottom_bc=None, top_bc=None) -> Mesh2D:
    """Unit-square mesh with the sinusoidal warp (MeshMetrics2D.jl:261-292)."""
    m = Mesh2D(x_left, x_right, y_bottom, y_top, nx, ny, left_bc, right_bc, bottom_bc, top_bc)
    m.wavy_amp = float(amp)
    return m
