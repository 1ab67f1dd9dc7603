"""Solution state containers (src/solvestate/SolutionState.jl, SolutionState2D.jl).

Layout is the reference's: ``u[j, e, c]`` (1D) / ``u[i, j, e, c]`` (2D) as a
Fortran-ordered numpy array, so a state uploads to the GPU as one copy.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .equations import EPS
from .mesh import Mesh1D, Mesh2D
from .operators import FROperators
from .scheme import DEFAULT_SCHEME, SchemeConfig


class SolutionState:
    """1D state: u[Np, Nel, Neq], time, mesh, operators, scheme."""

    dim = 1

    def __init__(self, mesh: Mesh1D, ops: FROperators, neq: int, scheme: SchemeConfig):
        self.mesh, self.ops, self.scheme = mesh, ops, scheme
        self.p = ops.p
        self.u = np.zeros((ops.p + 1, mesh.n_elements, neq), order="F")
        self.t = 0.0
        self._gpu = {}

    @property
    def neq(self) -> int:
        return self.u.shape[-1]


class SolutionState2D:
    """2D state: u[Np, Np, Nel, Neq] plus the mesh geometry choice."""

    dim = 2

    def __init__(self, mesh: Mesh2D, ops: FROperators, neq: int, scheme: SchemeConfig,
                 metrics: Optional[dict] = None, wavy_amp: Optional[float] = None):
        self.mesh, self.ops, self.scheme = mesh, ops, scheme
        self.p = ops.p
        n = ops.p + 1
        self.u = np.zeros((n, n, mesh.n_elements, neq), order="F")
        self.t = 0.0
        # geometry: caller metrics (MeshMetrics2D fields), analytic wavy, or affine
        self.metrics = metrics
        self.wavy_amp = wavy_amp if wavy_amp is not None else mesh.wavy_amp
        self._gpu = {}

    @property
    def neq(self) -> int:
        return self.u.shape[-1]


def allocate_state(mesh, ops: FROperators, neq: int, scheme: Optional[SchemeConfig] = None,
                   metrics: Optional[dict] = None, wavy_amp: Optional[float] = None):
    """allocate_state(mesh, ops, Val(Neq); scheme) (SolutionState.jl:25-48,
    SolutionState2D.jl:137-173)."""
    sch = scheme or SchemeConfig(ops.points, DEFAULT_SCHEME.flux, DEFAULT_SCHEME.time)
    if isinstance(mesh, Mesh1D):
        return SolutionState(mesh, ops, neq, sch)
    return SolutionState2D(mesh, ops, neq, sch, metrics=metrics, wavy_amp=wavy_amp)


def set_initial_condition_(state, f):
    """set_initial_condition!(state, f): f(x) (1D) or f(x, y) (2D) returns the
    conserved vector; vectorised numpy functions are accepted."""
    if state.dim == 1:
        X = state.mesh.physical_coords(state.ops)
        vals = np.asarray(f(X), dtype=np.float64)
    else:
        X, Y = state.mesh.physical_coords(state.ops)
        vals = np.asarray(f(X, Y), dtype=np.float64)
    state.u[...] = vals.reshape(state.u.shape)
    state.t = 0.0
    return state


def discrete_mass(state, c: int = 0) -> float:
    """GL-quadrature integral of component c (SolutionState.jl:80-90,
    SolutionState2D.jl:85-97); affine Jacobian."""
    w = state.ops.w
    if state.dim == 1:
        return float(np.sum(w[:, None] * state.mesh.J[None, :] * state.u[:, :, c]))
    m = state.mesh
    e = np.arange(m.n_elements)
    J = (m.Jx[e % m.nx] * m.Jy[e // m.nx])[None, None, :]
    return float(np.sum(w[:, None, None] * w[None, :, None] * np.abs(J) * state.u[:, :, :, c]))


def has_nonfinite(a) -> bool:
    return not bool(np.all(np.isfinite(a)))


def positivity_ok(eq, state, atol: float = 0.0) -> bool:
    """rho > atol and p > atol everywhere (Euler.jl:62-77, Euler2D.jl:153-163)."""
    rho = state.u[..., 0]
    p = eq.pressure(state.u)
    return bool(np.all((rho > atol) & (p > atol) & np.isfinite(rho) & np.isfinite(p)))


def solution_extrema(state, c: int = 0):
    v = state.u[..., c]
    return float(np.min(v)), float(np.max(v))
