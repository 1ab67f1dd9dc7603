"""ctypes front end of the C oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is a plain-C FP64 restatement of FRForge's residual + SSP-RK path
(``frforge_oracle.c``).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as the checker
or as the timed CPU baseline; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

POINTS = {"gl": 0, "gll": 1}
FLUX = {"rusanov": 0, "hllc": 1}
TIME = {"ssp_rk3": 0, "ssp_rk2": 1}
BC = {"periodic": 0, "transmissive": 1, "dirichlet": 2, "reflecting": 3, "xsplit": 4}
METHOD = {"null": 0, "persson": 1}
AV_FORM = {"conservative_br0": 0, "element_local_DD": 1}
STATUS = {0: "ok", 1: "diverged", 2: "max_steps"}


class OrcOps(C.Structure):
    _fields_ = [
        ("p", C.c_int), ("np", C.c_int), ("points", C.c_int),
        ("xi", C.c_double * 8), ("w", C.c_double * 8),
        ("D", C.c_double * 64),
        ("lL", C.c_double * 8), ("lR", C.c_double * 8),
        ("gLxi", C.c_double * 8), ("gRxi", C.c_double * 8),
        ("gL", C.c_double * 8), ("gR", C.c_double * 8),
        ("V", C.c_double * 64),
    ]

    def as_dict(self):
        n = self.np
        vec = lambda a: np.array(a[:n], dtype=np.float64)
        mat = lambda a: np.array(a[: n * n], dtype=np.float64).reshape(n, n, order="F")
        return {
            "p": self.p, "np": n, "points": self.points,
            "xi": vec(self.xi), "w": vec(self.w), "D": mat(self.D),
            "l_L": vec(self.lL), "l_R": vec(self.lR),
            "gL_xi": vec(self.gLxi), "gR_xi": vec(self.gRxi),
            "gL": vec(self.gL), "gR": vec(self.gR), "V": mat(self.V),
        }


class OrcBC(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("mode", C.c_int),
        ("state", C.c_double * 4), ("state_b", C.c_double * 4),
        ("x0", C.c_double), ("s0", C.c_double), ("s1", C.c_double), ("sdiv", C.c_double),
    ]


def make_bc(kind="periodic", state=None, state_b=None, x0=0.0, s0=0.0, s1=0.0, sdiv=1.0, mode=0):
    b = OrcBC()
    b.kind = BC[kind]
    b.mode = mode
    for i, v in enumerate(state or []):
        b.state[i] = v
    for i, v in enumerate(state_b or []):
        b.state_b[i] = v
    b.x0, b.s0, b.s1, b.sdiv = x0, s0, s1, sdiv
    return b


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, no GPU)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "frforge_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        dp, ip = C.POINTER(C.c_double), C.c_int
        L.orc_build_operators.argtypes = [ip, ip, C.POINTER(OrcOps)]
        L.orc_create_1d.restype = C.c_void_p
        L.orc_create_1d.argtypes = [ip, ip, ip, C.c_double, C.c_double, C.POINTER(OrcBC),
                                    C.POINTER(OrcBC), C.c_double, ip, ip, ip, ip,
                                    C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_create_2d.restype = C.c_void_p
        L.orc_create_2d.argtypes = [ip, ip, ip, ip, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.POINTER(OrcBC), C.c_void_p, ip, C.c_double,
                                    C.c_double, ip, ip, ip, ip, C.c_double, C.c_double,
                                    C.c_double, C.c_double]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_get_ops.argtypes = [C.c_void_p, C.POINTER(OrcOps)]
        L.orc_ndof.restype = C.c_size_t
        L.orc_ndof.argtypes = [C.c_void_p]
        L.orc_state.restype = dp
        L.orc_state.argtypes = [C.c_void_p]
        L.orc_get_time.restype = C.c_double
        L.orc_get_time.argtypes = [C.c_void_p]
        L.orc_set_time.argtypes = [C.c_void_p, C.c_double]
        L.orc_metric.restype = dp
        L.orc_metric.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_physical_coords.argtypes = [C.c_void_p, dp, dp]
        L.orc_set_threads.argtypes = [ip]
        L.orc_set_flux_override.argtypes = [C.c_void_p, ip, C.c_double]
        L.orc_set_trace_override.argtypes = [C.c_void_p, ip, C.c_double, C.c_double]
        L.orc_get_traces_1d.argtypes = [C.c_void_p, dp, dp]
        L.orc_residual.argtypes = [C.c_void_p, dp]
        L.orc_sense.argtypes = [C.c_void_p, dp]
        L.orc_compute_dt.restype = C.c_double
        L.orc_compute_dt.argtypes = [C.c_void_p, C.c_double]
        L.orc_step.argtypes = [C.c_void_p, C.c_double]
        L.orc_integrate.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                    C.c_int64, C.POINTER(C.c_int64)]
        L.orc_discrete_mass.restype = C.c_double
        L.orc_discrete_mass.argtypes = [C.c_void_p, ip]
        L.orc_positivity_ok.argtypes = [C.c_void_p]
        L.orc_has_nonfinite.argtypes = [dp, C.c_size_t]
        L.orc_solution_extrema.argtypes = [C.c_void_p, ip, dp, dp]
        for name in ("orc_ic_sod", "orc_ic_shu_osher", "orc_ic_smooth_2d"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_ic_density_wave_1d.argtypes = [C.c_void_p, C.c_double]
        L.orc_ic_two_state_1d.argtypes = [C.c_void_p, C.c_double, dp, dp]
        L.orc_ic_vortex_2d.argtypes = [C.c_void_p, C.c_double]
        L.orc_ic_four_quadrant_2d.argtypes = [C.c_void_p, C.c_double, C.c_double, dp, dp, dp, dp]
        L.orc_ic_uniform.argtypes = [C.c_void_p, dp]
        for name in ("orc_l2_error_vortex", "orc_l2_error_smooth_2d", "orc_l2_error_density_wave_1d"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_void_p, C.c_double]
        for name in ("orc_hllc_1d", "orc_rusanov_1d"):
            getattr(L, name).argtypes = [C.c_double, dp, dp, dp]
        for name in ("orc_hllc_2d", "orc_rusanov_2d"):
            getattr(L, name).argtypes = [C.c_double, dp, dp, C.c_double, C.c_double, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def build_operators(p: int, points: str = "gl") -> dict:
    o = OrcOps()
    if lib().orc_build_operators(p, POINTS[points], C.byref(o)) != 0:
        raise ValueError("invalid operator request")
    return o.as_dict()


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


class OracleSolver:
    """One reference-equivalent solve on the CPU (1D or 2D Euler)."""

    def __init__(self, handle, dim, np_, nel, neq, nx=None, ny=None):
        if not handle:
            raise ValueError("oracle rejected the configuration")
        self._h = C.c_void_p(handle)
        self.dim, self.np, self.nel, self.neq = dim, np_, nel, neq
        self.nx, self.ny = nx, ny

    @classmethod
    def one_d(cls, p=2, nel=64, xl=0.0, xr=1.0, left="transmissive", right="transmissive",
              left_state=None, right_state=None, gamma=1.4, points="gl", flux="rusanov",
              time="ssp_rk3", method="null", av_form="conservative_br0", kappa=4.0,
              s0_factor=-4.0, eps_floor=1e-16, c_av=0.1):
        bl = make_bc(left, left_state)
        br = make_bc(right, right_state)
        h = lib().orc_create_1d(p, POINTS[points], nel, xl, xr, C.byref(bl), C.byref(br), gamma,
                                FLUX[flux], TIME[time], METHOD[method], AV_FORM[av_form],
                                kappa, s0_factor, eps_floor, c_av)
        return cls(h, 1, p + 1, nel, 3)

    @classmethod
    def two_d(cls, p=2, nx=8, ny=8, xl=0.0, xr=1.0, yb=0.0, yt=1.0, bcs=None, solid=None,
              wavy=0, amp=0.05, gamma=1.4, points="gl", flux="rusanov", time="ssp_rk3",
              method="null", av_form="conservative_br0", kappa=4.0, s0_factor=-4.0,
              eps_floor=1e-16, c_av=0.1):
        if bcs is None:
            bcs = [make_bc("periodic") for _ in range(4)]
        arr = (OrcBC * 4)(*bcs)
        solid_ptr = None
        if solid is not None:
            solid_arr = np.ascontiguousarray(solid, dtype=np.uint8)
            solid_ptr = solid_arr.ctypes.data_as(C.c_void_p)
        h = lib().orc_create_2d(p, POINTS[points], nx, ny, xl, xr, yb, yt, arr, solid_ptr,
                                int(wavy), amp, gamma, FLUX[flux], TIME[time], METHOD[method],
                                AV_FORM[av_form], kappa, s0_factor, eps_floor, c_av)
        return cls(h, 2, p + 1, nx * ny, 4, nx, ny)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    # -- state ---------------------------------------------------------
    @property
    def shape(self):
        if self.dim == 1:
            return (self.np, self.nel, self.neq)
        return (self.np, self.np, self.nel, self.neq)

    @property
    def ndof(self) -> int:
        return int(lib().orc_ndof(self._h))

    @property
    def u(self) -> np.ndarray:
        """Live view of the state in the Julia column-major layout."""
        ptr = lib().orc_state(self._h)
        flat = np.ctypeslib.as_array(ptr, shape=(self.ndof,))
        return flat.reshape(self.shape, order="F")

    def set_state(self, u: np.ndarray) -> None:
        self.u[...] = np.asarray(u, dtype=np.float64).reshape(self.shape, order="F")

    @property
    def t(self) -> float:
        return lib().orc_get_time(self._h)

    @t.setter
    def t(self, v: float) -> None:
        lib().orc_set_time(self._h, float(v))

    def ops(self) -> dict:
        o = OrcOps()
        lib().orc_get_ops(self._h, C.byref(o))
        return o.as_dict()

    def metric(self, name: str) -> np.ndarray:
        ptr = lib().orc_metric(self._h, name.encode())
        if not ptr:
            raise KeyError(name)
        n = self.nel if name == "h_char" else (
            self.np * self.nel if name[:2] in ("nx", "ny", "sJ") else self.np * self.np * self.nel)
        a = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        if name == "h_char":
            return a
        if name[:2] in ("nx", "ny", "sJ"):
            return a.reshape(self.np, self.nel, order="F")
        return a.reshape(self.np, self.np, self.nel, order="F")

    def coords(self):
        n = self.ndof // self.neq
        x = np.zeros(n)
        y = np.zeros(n)
        lib().orc_physical_coords(self._h, _dp(x), _dp(y))
        if self.dim == 1:
            return x.reshape(self.np, self.nel, order="F")
        return (x.reshape(self.np, self.np, self.nel, order="F"),
                y.reshape(self.np, self.np, self.nel, order="F"))

    # -- hot path --------------------------------------------------------
    def set_flux_override(self, kind=None, alpha: float = 1.0) -> None:
        """A 1D method's numerical_flux_method override: None (the scheme's
        flux), "rusanov" (dissipation scaled by alpha) or "hllc"."""
        k = -1 if kind is None else {"rusanov": 0, "hllc": 1}[kind]
        lib().orc_set_flux_override(self._h, k, float(alpha))

    def set_trace_override(self, kind=None, p0: float = 1.0, p1: float = 1e-13) -> None:
        """A 1D method's extrapolate_interface! override: None (the Lagrange
        traces), "toward_mean" (p0 = theta) or "positivity" (p0 = eps_rho,
        p1 = eps_p)."""
        k = 0 if kind is None else {"toward_mean": 1, "positivity": 2}[kind]
        lib().orc_set_trace_override(self._h, k, float(p0), float(p1))

    def traces_1d(self):
        """(uL, uR) [nel, 3]: the traces the last residual's fluxes used."""
        tl, tr = np.zeros(self.nel * 3), np.zeros(self.nel * 3)
        lib().orc_get_traces_1d(self._h, _dp(tl), _dp(tr))
        return tl.reshape(self.nel, 3, order="F"), tr.reshape(self.nel, 3, order="F")

    def residual(self) -> np.ndarray:
        du = np.zeros(self.ndof)
        lib().orc_residual(self._h, _dp(du))
        return du.reshape(self.shape, order="F")

    def sense(self) -> np.ndarray:
        s = np.zeros(self.nel)
        lib().orc_sense(self._h, _dp(s))
        return s

    def compute_dt(self, cfl: float) -> float:
        return lib().orc_compute_dt(self._h, cfl)

    def step(self, dt: float) -> str:
        return STATUS[lib().orc_step(self._h, dt)]

    def integrate(self, t_final, cfl=0.2, dt=None, max_steps=10**7):
        n = C.c_int64(0)
        st = lib().orc_integrate(self._h, t_final, cfl, -1.0 if dt is None else float(dt),
                                 int(max_steps), C.byref(n))
        return {"status": STATUS[st], "n_steps": int(n.value), "t": self.t}

    # -- diagnostics -----------------------------------------------------
    def discrete_mass(self, c: int = 0) -> float:
        return lib().orc_discrete_mass(self._h, c)

    def positivity_ok(self) -> bool:
        return bool(lib().orc_positivity_ok(self._h))

    def has_nonfinite(self) -> bool:
        u = np.ascontiguousarray(self.u.ravel(order="F"))
        return bool(lib().orc_has_nonfinite(_dp(u), u.size))

    def extrema(self, c: int = 0):
        lo, hi = C.c_double(), C.c_double()
        lib().orc_solution_extrema(self._h, c, C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    # -- reference initial conditions --------------------------------------
    def ic_sod(self):
        lib().orc_ic_sod(self._h)

    def ic_shu_osher(self):
        lib().orc_ic_shu_osher(self._h)

    def ic_density_wave(self, t=0.0):
        lib().orc_ic_density_wave_1d(self._h, t)

    def ic_two_state(self, x0, primL, primR):
        a = np.asarray(primL, dtype=np.float64)
        b = np.asarray(primR, dtype=np.float64)
        lib().orc_ic_two_state_1d(self._h, x0, _dp(a), _dp(b))

    def ic_vortex(self, t=0.0):
        lib().orc_ic_vortex_2d(self._h, t)

    def ic_smooth_2d(self):
        lib().orc_ic_smooth_2d(self._h)

    def ic_four_quadrant(self, ne, nw, sw, se, x0=0.5, y0=0.5):
        arrs = [np.asarray(v, dtype=np.float64) for v in (ne, nw, sw, se)]
        lib().orc_ic_four_quadrant_2d(self._h, x0, y0, *[_dp(a) for a in arrs])

    def ic_uniform(self, prim):
        a = np.asarray(prim, dtype=np.float64)
        lib().orc_ic_uniform(self._h, _dp(a))

    def l2_error_vortex(self, t):
        return lib().orc_l2_error_vortex(self._h, t)

    def l2_error_smooth_2d(self, t):
        return lib().orc_l2_error_smooth_2d(self._h, t)

    def l2_error_density_wave(self, t):
        return lib().orc_l2_error_density_wave_1d(self._h, t)


def flux_1d(kind, gamma, uL, uR):
    out = np.zeros(3)
    a, b = np.asarray(uL, dtype=np.float64), np.asarray(uR, dtype=np.float64)
    getattr(lib(), f"orc_{kind}_1d")(gamma, _dp(a), _dp(b), _dp(out))
    return out


def flux_2d(kind, gamma, uL, uR, nx, ny):
    out = np.zeros(4)
    a, b = np.asarray(uL, dtype=np.float64), np.asarray(uR, dtype=np.float64)
    getattr(lib(), f"orc_{kind}_2d")(gamma, _dp(a), _dp(b), nx, ny, _dp(out))
    return out
