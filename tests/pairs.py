"""Matched oracle / GPU set-ups for the parity tests.

Each config builds the same mesh, scheme, method and initial state in the C
oracle (the checker) and in frforge_b200 (the product), so tests compare the
two on identical inputs.
"""
from __future__ import annotations

import numpy as np

import oracle as O
import frforge_b200 as F

GAMMA = 1.4


def prim2cons2(r, u, v, p):
    E = p / (GAMMA - 1.0) + 0.5 * r * (u * u + v * v)
    return np.stack([r, r * u, r * v, E], axis=-1)


def prim2cons1(r, u, p):
    E = p / (GAMMA - 1.0) + 0.5 * r * u * u
    return np.stack([r, r * u, E], axis=-1)


def splitmix64(seed: int):
    """SplitMix64 stream (Steele, Lea, Flood 2014) -> uniform doubles in [0,1)."""
    state = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        yield (z >> 11) * (1.0 / 9007199254740992.0)


BC_MAP = {"periodic": F.PeriodicBC, "transmissive": F.TransmissiveBC, "reflecting": F.ReflectingBC}


def _gpu_bc(spec):
    if isinstance(spec, tuple) and spec[0] == "dirichlet":
        return F.DirichletBC(list(spec[1]))
    return BC_MAP[spec]()


def _orc_bc(spec):
    if isinstance(spec, tuple) and spec[0] == "dirichlet":
        return O.make_bc("dirichlet", list(spec[1]))
    return O.make_bc(spec)


def method_objects(method: str, c_av: float, av_form: str):
    if method == "null":
        return F.NullCapturing(), dict(method="null")
    return (F.PerssonAVMethod(c_av=c_av, av_form=av_form),
            dict(method="persson", c_av=c_av, av_form=av_form))


def pair_2d(p=3, nx=8, ny=8, points="gl", flux="rusanov", time="ssp_rk3", method="null", c_av=0.1,
            av_form="conservative_br0", bcs=("periodic",) * 4, solid=None, wavy=0, amp=0.05,
            xl=0.0, xr=1.0, yb=0.0, yt=1.0, gpu_metrics=False, caller_ops=False):
    orc_method = method_objects(method, c_av, av_form)[1]
    orc = O.OracleSolver.two_d(p=p, nx=nx, ny=ny, xl=xl, xr=xr, yb=yb, yt=yt,
                               bcs=[_orc_bc(b) for b in bcs], solid=solid, wavy=wavy, amp=amp,
                               points=points, flux=flux, time=time, **orc_method)
    mesh = F.Mesh2D(xl, xr, yb, yt, nx, ny, *[_gpu_bc(b) for b in bcs], solid=solid)
    ops = F.build_operators(p, points)
    metrics = None
    if gpu_metrics:
        metrics = {n: orc.metric(n) for n in ("x_xi", "x_eta", "y_xi", "y_eta", "J", "nx_W", "ny_W",
                                              "sJ_W", "nx_E", "ny_E", "sJ_E", "nx_S", "ny_S", "sJ_S",
                                              "nx_N", "ny_N", "sJ_N", "h_char")}
    state = F.allocate_state(mesh, ops, 4, scheme=F.SchemeConfig(points, flux, time), metrics=metrics,
                             wavy_amp=amp if (wavy == 1 and not gpu_metrics) else None)
    gmethod = method_objects(method, c_av, av_form)[0]
    solve = F.GpuSolve(state, F.Euler2D(GAMMA), gmethod, caller_ops=orc.ops() if caller_ops else None)
    return orc, state, solve


def pair_1d(p=3, nel=32, points="gl", flux="rusanov", time="ssp_rk3", method="null", c_av=0.1,
            av_form="conservative_br0", left="transmissive", right="transmissive", xl=0.0, xr=1.0,
            caller_ops=False):
    orc_method = method_objects(method, c_av, av_form)[1]
    lk, ls = (left[0], list(left[1])) if isinstance(left, tuple) else (left, None)
    rk, rs = (right[0], list(right[1])) if isinstance(right, tuple) else (right, None)
    orc = O.OracleSolver.one_d(p=p, nel=nel, xl=xl, xr=xr, left=lk, right=rk, left_state=ls,
                               right_state=rs, points=points, flux=flux, time=time, **orc_method)
    mesh = F.Mesh1D(xl, xr, nel, _gpu_bc(left), _gpu_bc(right))
    ops = F.build_operators(p, points)
    state = F.allocate_state(mesh, ops, 3, scheme=F.SchemeConfig(points, flux, time))
    gmethod = method_objects(method, c_av, av_form)[0]
    solve = F.GpuSolve(state, F.Euler1D(GAMMA), gmethod, caller_ops=orc.ops() if caller_ops else None)
    return orc, state, solve


def four_quadrant_state(orc, seed=20261203, x0=0.5, y0=0.5, states=None, jump_scale=1.0):
    """Seeded four-quadrant Riemann IC (riemann2d_ic quadrant rule,
    Cases2D_Riemann.jl:33-51); draws in the order ne, nw, sw, se; each state's
    deviation from the mean of the four is scaled by jump_scale."""
    if states is None:
        g = splitmix64(seed)
        states = []
        for _ in range(4):
            r = 0.1 + 1.4 * next(g)
            u = -0.8 + 1.6 * next(g)
            v = -0.8 + 1.6 * next(g)
            p = 0.05 + 1.45 * next(g)
            states.append(np.array((r, u, v, p)))
        m = sum(states) / 4.0
        states = [tuple(m + jump_scale * (s - m)) for s in states]
    x, y = orc.coords()
    ne, nw, sw, se = [np.array(s) for s in states]
    P = np.where(((x >= x0) & (y >= y0))[..., None], ne,
                 np.where(((x < x0) & (y >= y0))[..., None], nw,
                          np.where(((x < x0) & (y < y0))[..., None], sw, se)))
    return prim2cons2(P[..., 0], P[..., 1], P[..., 2], P[..., 3])


def smooth_state_2d(orc, seed=7, amp=0.2):
    x, y = orc.coords()
    g = splitmix64(seed)
    ph = [2 * np.pi * next(g) for _ in range(4)]
    r = 1.0 + amp * np.sin(2 * np.pi * (x + y) + ph[0])
    u = 0.5 + 0.3 * np.sin(2 * np.pi * x + ph[1])
    v = -0.3 + 0.2 * np.cos(2 * np.pi * y + ph[2])
    p = 1.0 + 0.1 * np.sin(2 * np.pi * (x - y) + ph[3])
    return prim2cons2(r, u, v, p)


def rel_linf(got, ref):
    scale = np.max(np.abs(ref))
    err = np.max(np.abs(got - ref))
    return err / scale if scale > 0 else err
