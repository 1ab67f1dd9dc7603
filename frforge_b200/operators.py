"""FROperators: reference-element operators (src/fr/Operators.jl:62-104).

Built by the library's host code (``frg_build_operators``); callers that
already hold the reference's tables can pass them to a solve instead.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class FROperators:
    p: int
    points: str
    xi: np.ndarray
    w: np.ndarray
    D: np.ndarray
    l_L: np.ndarray
    l_R: np.ndarray
    gL_xi: np.ndarray
    gR_xi: np.ndarray
    gL: np.ndarray
    gR: np.ndarray
    V_legendre: np.ndarray

    @property
    def np_(self) -> int:
        return self.p + 1


def n_points(ops: FROperators) -> int:
    return len(ops.xi)


def build_operators(p: int, points: str = "gl") -> FROperators:
    """build_operators(p; points) (Operators.jl:85-104)."""
    if p < 1 or p > 5:
        raise ValueError("p must be in 1..5 on the GPU path")
    if points not in L.POINTS:
        raise ValueError(f"points must be :gl or :gll, got {points}")
    n = p + 1
    a = {k: np.zeros(n) for k in ("xi", "w", "l_L", "l_R", "gL_xi", "gR_xi", "gL", "gR")}
    D = np.zeros(n * n)
    V = np.zeros(n * n)
    L.check(L.load().frg_build_operators(p, L.POINTS[points], L.dptr(a["xi"]), L.dptr(a["w"]),
                                         L.dptr(D), L.dptr(a["l_L"]), L.dptr(a["l_R"]),
                                         L.dptr(a["gL_xi"]), L.dptr(a["gR_xi"]), L.dptr(a["gL"]),
                                         L.dptr(a["gR"]), L.dptr(V)), what="build_operators")
    return FROperators(p=p, points=points, D=D.reshape(n, n, order="F"),
                       V_legendre=V.reshape(n, n, order="F"), **a)
