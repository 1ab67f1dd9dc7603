"""Seeded synthetic workloads (no public suite is involved).

All draws come from one SplitMix64 stream (Steele, Lea & Flood 2014) in a
fixed order, default seed 20261203, so the oracle, the GPU and the CPU
baseline see identical inputs.

* c1: 1D Euler, 256 elements on [0,1], GL P=3, Rusanov, SSP-RK3, Persson AV
  (c_av 0.1, BR0), transmissive; two-state Riemann IC at x=0.5 with left then
  right (rho, u, p) drawn rho~U[0.1,1], u~U[-0.5,0.5], p~U[0.1,1]; CFL 0.1.
* c2: 2D periodic [0,1]^2, 128^2 affine quads, GL P=4, Rusanov, SSP-RK3,
  Persson AV; rho = 1 + 0.2 sin(2 pi (x+y) + phi), phi~U[0,2pi), u=v=p=1.
* c3: 2D [0,1]^2, 512^2 quads, GL P=3, HLLC, SSP-RK3, Persson AV (c_av 0.1,
  BR0), transmissive, CFL 0.1; four-quadrant piecewise-constant IC split at
  (0.5, 0.5) with the quadrant rule of riemann2d_ic
  (src/verification/Cases2D_Riemann.jl:33-51).  The four (rho,u,v,p) states
  are drawn rho~U[0.1,1.5], u,v~U[-0.8,0.8], p~U[0.05,1.5] in the order
  ne, nw, sw, se, and then each state's deviation from the mean of the four
  is scaled by ``jump_scale`` = 0.25: with the unscaled draws the reference
  scheme itself (P=3 FR + HLLC + Persson AV, no positivity limiter) reaches
  negative density and returns :diverged within 40 steps for every seed
  tried, which would leave nothing to time.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Iterator, List, Tuple

import numpy as np

DEFAULT_SEED = 20261203


def splitmix64(seed: int) -> Iterator[float]:
    """Uniform doubles in [0, 1) from SplitMix64 (53-bit mantissa)."""
    state = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        yield (z >> 11) * (1.0 / 9007199254740992.0)


def uniform(g: Iterator[float], lo: float, hi: float) -> float:
    return lo + (hi - lo) * next(g)


def four_quadrant_states(seed: int = DEFAULT_SEED, jump_scale: float = 0.25) -> List[Tuple[float, ...]]:
    g = splitmix64(seed)
    st = []
    for _ in range(4):
        st.append(np.array([uniform(g, 0.1, 1.5), uniform(g, -0.8, 0.8), uniform(g, -0.8, 0.8),
                            uniform(g, 0.05, 1.5)]))
    m = sum(st) / 4.0
    return [tuple(m + jump_scale * (s - m)) for s in st]


def four_quadrant_ic(X, Y, states, gamma=1.4, x0=0.5, y0=0.5) -> np.ndarray:
    """Conserved state [..., 4] of the four-quadrant rule (riemann2d_ic)."""
    ne, nw, sw, se = [np.asarray(s) for s in states]
    P = np.where(((X >= x0) & (Y >= y0))[..., None], ne,
                 np.where(((X < x0) & (Y >= y0))[..., None], nw,
                          np.where(((X < x0) & (Y < y0))[..., None], sw, se)))
    r, u, v, p = P[..., 0], P[..., 1], P[..., 2], P[..., 3]
    E = p / (gamma - 1.0) + 0.5 * r * (u * u + v * v)
    return np.stack([r, r * u, r * v, E], axis=-1)


def two_state_1d(seed: int = DEFAULT_SEED):
    g = splitmix64(seed)
    L = (uniform(g, 0.1, 1.0), uniform(g, -0.5, 0.5), uniform(g, 0.1, 1.0))
    R = (uniform(g, 0.1, 1.0), uniform(g, -0.5, 0.5), uniform(g, 0.1, 1.0))
    return L, R


@dataclass
class Workload2D:
    name: str
    n: int
    p: int
    flux: str
    method: str
    c_av: float
    periodic: bool
    cfl: float
    steps: int
    seed: int = DEFAULT_SEED
    jump_scale: float = 0.25

    @property
    def ndof(self) -> int:
        return self.n * self.n * (self.p + 1) ** 2 * 4

    def build(self, F):
        """(state, method) for the frforge_b200 module F, IC filled in."""
        bc = F.PeriodicBC if self.periodic else F.TransmissiveBC
        mesh = F.Mesh2D(0.0, 1.0, 0.0, 1.0, self.n, self.n, bc(), bc(), bc(), bc())
        ops = F.build_operators(self.p)
        st = F.allocate_state(mesh, ops, 4, scheme=F.SchemeConfig("gl", self.flux, "ssp_rk3"))
        X, Y = mesh.physical_coords(ops)
        st.u[...] = self.initial_state(X, Y)
        m = F.PerssonAVMethod(c_av=self.c_av) if self.method == "persson_av" else F.NullCapturing()
        return st, m

    def initial_state(self, X, Y) -> np.ndarray:
        if self.name == "c2":
            g = splitmix64(self.seed)
            phi = uniform(g, 0.0, 2 * math.pi)
            r = 1.0 + 0.2 * np.sin(2 * math.pi * (X + Y) + phi)
            one = np.ones_like(r)
            return np.stack([r, r, r, one / (1.4 - 1.0) + 0.5 * r * (1.0 * 1.0 + 1.0 * 1.0)], axis=-1)
        return four_quadrant_ic(X, Y, four_quadrant_states(self.seed, self.jump_scale))


@dataclass
class Workload1D:
    name: str
    nel: int
    p: int
    flux: str
    method: str
    c_av: float
    cfl: float
    steps: int
    seed: int = DEFAULT_SEED

    @property
    def ndof(self) -> int:
        return self.nel * (self.p + 1) * 3

    def build(self, F):
        """(state, method) for the frforge_b200 module F, IC filled in."""
        mesh = F.Mesh1D(0.0, 1.0, self.nel, F.TransmissiveBC(), F.TransmissiveBC())
        ops = F.build_operators(self.p)
        st = F.allocate_state(mesh, ops, 3, scheme=F.SchemeConfig("gl", self.flux, "ssp_rk3"))
        st.u[...] = self.initial_state(mesh.physical_coords(ops))
        m = F.PerssonAVMethod(c_av=self.c_av) if self.method == "persson_av" else F.NullCapturing()
        return st, m

    def initial_state(self, x, gamma: float = 1.4) -> np.ndarray:
        """Two states split at x = 0.5 (left for x < 0.5, as sod_ic)."""
        (rL, uL, pL), (rR, uR, pR) = two_state_1d(self.seed)
        left = x < 0.5
        r = np.where(left, rL, rR)
        u = np.where(left, uL, uR)
        p = np.where(left, pL, pR)
        return np.stack([r, r * u, p / (gamma - 1.0) + 0.5 * r * u * u], axis=-1)


C1 = Workload1D("c1", 256, 3, "rusanov", "persson_av", 0.1, 0.1, 2000)
C2 = Workload2D("c2", 128, 4, "rusanov", "persson_av", 0.1, True, 0.1, 500)
C3 = Workload2D("c3", 512, 3, "hllc", "persson_av", 0.1, False, 0.1, 1000)
WORKLOADS = {"c2": C2, "c3": C3}


def c4_instances(seed: int = DEFAULT_SEED, count: int = 64, steps: int = 200) -> List[Workload2D]:
    """The batched workload: ``count`` independent 2D solves drawn from one
    SplitMix64 stream, per instance in this order: n = round(exp(U[ln 16,
    ln 256])) elements per side, P ~ U{1..5}, flux HLLC or Rusanov with
    probability 1/2 each, c_av = 0.1 * U[0.5, 2].  Even instances are periodic
    density waves, odd ones transmissive four-quadrant problems; each IC has
    its own seed (seed + 1 + index).  Every instance runs ``steps`` SSP-RK3
    steps at CFL 0.1 with Persson AV (BR0).  About 0.75 M elements and 54 M
    DOF in total at the default size."""
    g = splitmix64(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(uniform(g, math.log(16.0), math.log(256.0)))))
        p = 1 + min(int(5.0 * next(g)), 4)
        flux = "hllc" if next(g) < 0.5 else "rusanov"
        c_av = 0.1 * uniform(g, 0.5, 2.0)
        periodic = i % 2 == 0
        out.append(Workload2D("c2" if periodic else "c3", n, p, flux, "persson_av", c_av, periodic, 0.1,
                              steps, seed=seed + 1 + i))
    return out


@dataclass
class Request:
    """One served solve of the served trace."""
    arrival: float  # seconds after the trace start
    dim: int
    n: int  # elements per side (2D) or elements (1D)
    p: int
    flux: str
    periodic: bool  # density wave (True) or Riemann problem (False); periodic domain
    wavy: bool  # 2D: sinusoidal mesh warp, amplitude 0.05, analytic metrics
    t_final: float
    seed: int
    cfl: float = 0.1

    @property
    def ndof(self) -> int:
        return self.n * self.n * (self.p + 1) ** 2 * 4 if self.dim == 2 else self.n * (self.p + 1) * 3

    def ic(self) -> dict:
        """The request's initial condition as a device-side case IC
        (keyword arguments of frforge_b200._lib.make_ic): the same state
        build() evaluates on the host."""
        g = splitmix64(self.seed)
        if self.periodic:
            phi = uniform(g, 0.0, 2 * math.pi)
            prim = [(1.0, 1.0, 1.0)] if self.dim == 1 else [(1.0, 1.0, 1.0, 1.0)]
            return dict(kind="density_wave", prim=prim, amp=0.2, phase=phi)
        if self.dim == 1:
            L, R = two_state_1d(self.seed)
            m = [(a + b) / 2.0 for a, b in zip(L, R)]
            L = [mm + 0.25 * (a - mm) for mm, a in zip(m, L)]
            R = [mm + 0.25 * (b - mm) for mm, b in zip(m, R)]
            return dict(kind="two_state", prim=[L, R], x0=0.5)
        return dict(kind="four_quadrant", prim=four_quadrant_states(self.seed, 0.25), x0=0.5, y0=0.5)

    def build(self, F, fill: bool = True):
        """(state, eq, method) for the frforge_b200 module F, IC filled in
        (fill=False: mesh and scheme only, the state left zero, for a
        device-side IC)."""
        g = splitmix64(self.seed)
        ops = F.build_operators(self.p)
        method = F.PerssonAVMethod(c_av=0.1)
        bc = F.PeriodicBC
        if self.dim == 1:
            mesh = F.Mesh1D(0.0, 1.0, self.n, bc(), bc())
            st = F.allocate_state(mesh, ops, 3, scheme=F.SchemeConfig("gl", self.flux, "ssp_rk3"))
            if not fill:
                return st, F.Euler1D(1.4), method
            X = mesh.physical_coords(ops)
            if self.periodic:
                phi = uniform(g, 0.0, 2 * math.pi)
                r, u, p = 1.0 + 0.2 * np.sin(2 * math.pi * X + phi), 1.0 + 0 * X, 1.0 + 0 * X
            else:
                L, R = two_state_1d(self.seed)
                m = [(a + b) / 2.0 for a, b in zip(L, R)]
                L = [mm + 0.25 * (a - mm) for mm, a in zip(m, L)]
                R = [mm + 0.25 * (b - mm) for mm, b in zip(m, R)]
                r = np.where(X < 0.5, L[0], R[0])
                u = np.where(X < 0.5, L[1], R[1])
                p = np.where(X < 0.5, L[2], R[2])
            st.u[...] = np.stack([r, r * u, p / (1.4 - 1.0) + 0.5 * r * u * u], axis=-1)
            return st, F.Euler1D(1.4), method
        if self.wavy:
            mesh = F.make_wavy_mesh2d(self.n, self.n, amp=0.05, left_bc=bc(), right_bc=bc(), bottom_bc=bc(),
                                      top_bc=bc())
        else:
            mesh = F.Mesh2D(0.0, 1.0, 0.0, 1.0, self.n, self.n, bc(), bc(), bc(), bc())
        st = F.allocate_state(mesh, ops, 4, scheme=F.SchemeConfig("gl", self.flux, "ssp_rk3"))
        if not fill:
            return st, F.Euler2D(1.4), method
        X, Y = mesh.physical_coords(ops)
        w = Workload2D("c2" if self.periodic else "c3", self.n, self.p, self.flux, "persson_av", 0.1,
                       self.periodic, self.cfl, 0, seed=self.seed)
        st.u[...] = w.initial_state(X, Y)
        return st, F.Euler2D(1.4), method


def served_trace(seed: int = DEFAULT_SEED, count: int = 32, rate: float = 200.0, n2d=(16, 384),
                 n1d=(128, 4096), t_final=(0.05, 0.25)) -> List[Request]:
    """The served workload: ``count`` requests with Poisson arrivals at
    ``rate`` per second, drawn from one SplitMix64 stream, per request in this
    order: inter-arrival Exp(rate), 1D or 2D with probability 1/2, size (2D
    n ~ U{n2d}, 1D Ne ~ U{n1d}), P ~ U{1..5}, flux HLLC or Rusanov, density
    wave or Riemann problem, for 2D a wavy mesh (amplitude 0.05) with
    probability 1/4, t_final ~ U[t_final].  Persson AV (BR0, c_av 0.1),
    SSP-RK3, CFL 0.1, periodic domains.  Riemann states are drawn as for the
    single-solve workloads and their jumps about the mean scaled by 0.25
    (unscaled, the scheme without a limiter loses positivity); 2D Riemann
    problems use the four-quadrant rule.  Domains are periodic because the
    transmissive boundary of the reference scheme has a growing mode at high
    P (a 1e-12 perturbation at the right boundary of a P=5 Rusanov mesh grows
    to 5e-4 in 2000 steps in the oracle), so whether a long transmissive run
    diverges depends on rounding noise."""
    g = splitmix64(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += -math.log(1.0 - next(g)) / rate
        dim = 2 if next(g) < 0.5 else 1
        lo, hi = n2d if dim == 2 else n1d
        n = lo + min(int((hi - lo + 1) * next(g)), hi - lo)
        p = 1 + min(int(5.0 * next(g)), 4)
        flux = "hllc" if next(g) < 0.5 else "rusanov"
        periodic = next(g) < 0.5
        wavy = dim == 2 and next(g) < 0.25
        tf = uniform(g, t_final[0], t_final[1])
        out.append(Request(t, dim, n, p, flux, periodic, wavy, tf, seed + 1000 + i))
    return out
