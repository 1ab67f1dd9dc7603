"""Capturing-method hook surface and registry (src/capturing/Interfaces.jl,
PerssonAV.jl, src/methods/Registry.jl, ScaledPersson.jl).

A method is an object with the reference's six hooks.  The GPU library
implements the default hooks, the Persson modal sensor and both dissipation
forms; ``gpu_spec()`` turns a method into the solve descriptor fields.  A
subclass that overrides a hook with host code has no device form: building
its descriptor raises ``UnsupportedHookError`` instead of silently running
something else.
"""
from __future__ import annotations

from typing import Callable, Dict

from ._lib import FRG_ERR_UNSUPPORTED_HOOK, UnsupportedHookError

HOOKS = ("preprocess_state_", "extrapolate_interface_", "numerical_flux_method", "sense_",
         "apply_dissipation_", "post_step_")


class AbstractCapturingMethod:
    """Hook defaults are identities (Interfaces.jl:43-92).  The GPU runs them
    as part of the fused stage kernel; calling them on the host is not part
    of the GPU path."""

    def preprocess_state_(self, u_work, state, eq):
        u_work[...] = state.u
        return u_work

    def extrapolate_interface_(self, traces, u_work, state, eq):
        raise NotImplementedError("interface extrapolation runs inside the GPU stage kernel")

    def numerical_flux_method(self, eq, uL, uR):
        return None

    def sense_(self, sigma, u_work, state, eq):
        sigma[...] = 0.0
        return sigma

    def apply_dissipation_(self, du, sigma, u_work, state, eq):
        return du

    def post_step_(self, state, eq):
        return None

    # -- GPU descriptor ----------------------------------------------------
    _gpu_base: tuple = ()

    def gpu_spec(self) -> dict:
        for base in type(self).__mro__:
            if base in _GPU_CLASSES:
                known = base
                break
        else:
            raise UnsupportedHookError(FRG_ERR_UNSUPPORTED_HOOK,
                                       f"{type(self).__name__} has no GPU implementation")
        device = getattr(self, "gpu_hooks", {}) or {}
        for h in HOOKS:
            if getattr(type(self), h) is not getattr(known, h):
                # an overridden hook runs on the GPU only if the method names a
                # registered device implementation for it
                if h.rstrip("_") not in device:
                    raise UnsupportedHookError(
                        FRG_ERR_UNSUPPORTED_HOOK,
                        f"{type(self).__name__}.{h} overrides a hook the GPU path cannot run")
        spec = known._spec(self)
        spec["hooks"] = {slot: (name, tuple(params)) for slot, (name, params) in device.items()}
        return spec

    @staticmethod
    def _spec(m) -> dict:
        return {"method": "null", "av_form": "conservative_br0", "kappa": 4.0, "s0_factor": -4.0,
                "eps_floor": 1e-16, "c_av": 0.0}


class NullCapturing(AbstractCapturingMethod):
    """Default method: no sensor, no artificial viscosity."""

    def method_params(self):
        return {"method": "null"}


class PerssonSensor:
    """Persson-Peraire modal sensor parameters (PerssonAV.jl:8-27)."""

    def __init__(self, kappa=4.0, s0_factor=-4.0, eps_floor=1e-16):
        self.kappa, self.s0_factor, self.eps_floor = float(kappa), float(s0_factor), float(eps_floor)


class ElementArtificialViscosity:
    """eps_e = c_av * sigma_e * (h_e/p) * lambda_e (PerssonAV.jl:30-49)."""

    def __init__(self, c_av=0.1, av_form="conservative_br0"):
        if av_form not in ("conservative_br0", "element_local_DD"):
            raise ValueError(f"Unsupported av_form={av_form}")
        self.c_av, self.av_form = float(c_av), av_form


class PerssonAVMethod(AbstractCapturingMethod):
    """Persson modal sensor + element AV (PerssonAV.jl:53-100); the code
    default c_av is 0.1 (PerssonAV.jl:60, :72-77)."""

    def __init__(self, kappa=4.0, s0_factor=-4.0, c_av=0.1, av_form="conservative_br0"):
        self.sensor = PerssonSensor(kappa, s0_factor)
        self.dissip = ElementArtificialViscosity(c_av, av_form)

    def sense_(self, sigma, u_work, state, eq):  # runs on the GPU (see gpu.sense_)
        raise NotImplementedError("the Persson sensor runs in the GPU stage kernel; use frforge_b200.sense_")

    def apply_dissipation_(self, du, sigma, u_work, state, eq):
        raise NotImplementedError("artificial viscosity runs in the GPU stage kernel")

    def method_params(self):
        return {"κ": self.sensor.kappa, "s0_factor": self.sensor.s0_factor,
                "c_av": self.dissip.c_av, "av_form": self.dissip.av_form, "method": "persson_av"}

    @staticmethod
    def _spec(m) -> dict:
        return {"method": "persson", "av_form": m.dissip.av_form, "kappa": m.sensor.kappa,
                "s0_factor": m.sensor.s0_factor, "eps_floor": m.sensor.eps_floor,
                "c_av": m.dissip.c_av}


class ScaledPerssonMethod(AbstractCapturingMethod):
    """Persson AV with c_av = 0.5 forwarding every hook to the inner method
    (src/methods/ScaledPersson.jl:15-62)."""

    def __init__(self, kappa=4.0, s0_factor=-4.0, c_av=0.5, av_form="conservative_br0"):
        self.inner = PerssonAVMethod(kappa, s0_factor, c_av, av_form)

    def method_params(self):
        p = self.inner.method_params()
        p["method"] = "scaled_persson"
        p["note"] = "example inventable method; elevated c_av over baseline persson_av"
        return p

    @staticmethod
    def _spec(m) -> dict:
        return m.inner.gpu_spec()


class PositivityPreservingPersson(PerssonAVMethod):
    """Persson AV plus the Zhang-Shu positivity-preserving scaling after
    every step: a capturing method that overrides post_step!
    (Interfaces.jl:88-91) and names the device implementation of that hook,
    so it runs on the GPU (frg_hooks.cu); post_step_ is the host
    restatement (frforge_b200.limiters)."""

    def __init__(self, kappa=4.0, s0_factor=-4.0, c_av=0.1, av_form="conservative_br0", eps_rho=1e-13,
                 eps_p=1e-13):
        super().__init__(kappa, s0_factor, c_av, av_form)
        self.eps_rho, self.eps_p = float(eps_rho), float(eps_p)
        self.gpu_hooks = {"post_step": ("positivity_zhang_shu", (self.eps_rho, self.eps_p))}

    def post_step_(self, state, eq):
        from .limiters import zhang_shu_limit_

        zhang_shu_limit_(state, eq, self.eps_rho, self.eps_p)
        return None

    def method_params(self):
        p = super().method_params()
        p.update({"method": "persson_av_positive", "eps_rho": self.eps_rho, "eps_p": self.eps_p})
        return p


class PositivityPreprocessPersson(PerssonAVMethod):
    """Persson AV whose preprocess_state! (Interfaces.jl:41-46) limits the
    work state the residual is evaluated on: u_work is the Zhang-Shu
    positivity-preserving scaling of the stage state, while the SSP-RK
    combination keeps the stage state itself.  A src/methods-style plugin
    that names the device implementation of the hook
    ("preprocess_positivity_zhang_shu", frg_hooks.cu), so it runs on the GPU;
    preprocess_state_ is the host restatement (frforge_b200.limiters)."""

    def __init__(self, kappa=4.0, s0_factor=-4.0, c_av=0.1, av_form="conservative_br0", eps_rho=1e-13,
                 eps_p=1e-13):
        super().__init__(kappa, s0_factor, c_av, av_form)
        self.eps_rho, self.eps_p = float(eps_rho), float(eps_p)
        self.gpu_hooks = {"preprocess_state": ("preprocess_positivity_zhang_shu", (self.eps_rho, self.eps_p))}

    def preprocess_state_(self, u_work, state, eq):
        import copy

        from .limiters import zhang_shu_limit_

        u_work[...] = state.u
        work = copy.copy(state)
        work.u = u_work
        zhang_shu_limit_(work, eq, self.eps_rho, self.eps_p)
        return u_work

    def method_params(self):
        p = super().method_params()
        p.update({"method": "persson_av_preprocess_positive", "eps_rho": self.eps_rho, "eps_p": self.eps_p})
        return p


class FluxOverridePersson(PerssonAVMethod):
    """Persson AV whose numerical_flux_method (Interfaces.jl:73-76) replaces
    the scheme's 1D interface flux: flux="rusanov" gives the Rusanov flux
    with its dissipation scaled by alpha, 1/2 (F(uL) + F(uR)) - 1/2 alpha
    lambda (uR - uL) (alpha = 1: Rusanov.jl:10-25), flux="hllc" the HLLC
    flux.  A src/methods-style plugin: it names the device implementation of
    the hook ("flux_rusanov" / "flux_hllc", frg_hooks.cu), so it runs on the
    GPU.  As in the reference, only the 1D residual consults the override."""

    def __init__(self, flux="rusanov", alpha=1.0, kappa=4.0, s0_factor=-4.0, c_av=0.1,
                 av_form="conservative_br0"):
        super().__init__(kappa, s0_factor, c_av, av_form)
        if flux not in ("rusanov", "hllc"):
            raise ValueError("flux must be 'rusanov' or 'hllc'")
        self.flux, self.alpha = flux, float(alpha)
        self.gpu_hooks = {"numerical_flux_method": (f"flux_{flux}", (self.alpha,) if flux == "rusanov" else ())}

    def numerical_flux_method(self, eq, uL, uR):
        """Host restatement (1D Euler, conserved (rho, rho u, E))."""
        import numpy as np

        if self.flux == "hllc":
            raise NotImplementedError("the HLLC override is evaluated by the GPU stage kernel")
        uL, uR = np.asarray(uL, dtype=np.float64), np.asarray(uR, dtype=np.float64)

        def flux(U):
            u = U[1] / U[0]
            r = max(U[0], np.finfo(np.float64).eps)
            p = (eq.gamma - 1.0) * (U[2] - 0.5 * r * (U[1] / r) ** 2)
            return np.array([U[1], U[1] * u + p, (U[2] + p) * u]), abs(U[1] / r) + np.sqrt(
                eq.gamma * max(p, np.finfo(np.float64).eps) / r)

        fL, sL = flux(uL)
        fR, sR = flux(uR)
        lam = self.alpha * max(sL, sR)
        return 0.5 * (fL + fR) - 0.5 * lam * (uR - uL)

    def method_params(self):
        p = super().method_params()
        p.update({"method": "persson_av_flux_override", "flux": self.flux, "alpha": self.alpha})
        return p


def _root01(a, b, c):
    """Smallest root in [0, 1] of a t^2 + b t + c (c > 0 >= a + b + c), the
    stable quadratic formula of the device limiter."""
    import math

    if abs(a) < 1e-300:
        return min(max(-c / b, 0.0), 1.0) if b != 0.0 else 0.0
    disc = max(b * b - 4.0 * a * c, 0.0)
    q = -0.5 * (b + math.copysign(math.sqrt(disc), b))
    r1, r2 = q / a, (c / q if q != 0.0 else 2.0)
    t = 1.0
    for r in (r1, r2):
        if 0.0 <= r <= 1.0:
            t = min(t, r)
    return t


class TraceOverridePersson(PerssonAVMethod):
    """Persson AV whose extrapolate_interface! (Interfaces.jl:49-71, "Override
    for hybrid reconstruction") replaces the Lagrange traces that the 1D
    interface fluxes use: kind="toward_mean" pulls each element's two traces
    toward its mean, ubar + theta (ell . u - ubar) (theta = 1: the default
    traces, theta = 0: first order); kind="positivity" applies the
    Zhang-Shu scaling to them (density >= eps_rho, then pressure >= eps_p).
    A src/methods-style plugin naming the device implementation of the hook
    ("traces_toward_mean" / "traces_positivity_zhang_shu", frg_hooks.cu).
    As in the reference, only the 1D residual calls it, and the BR0
    dissipation keeps the Lagrange traces."""

    def __init__(self, kind="toward_mean", theta=1.0, eps_rho=1e-13, eps_p=1e-13, kappa=4.0, s0_factor=-4.0,
                 c_av=0.1, av_form="conservative_br0"):
        super().__init__(kappa, s0_factor, c_av, av_form)
        if kind not in ("toward_mean", "positivity"):
            raise ValueError("kind must be 'toward_mean' or 'positivity'")
        self.kind, self.theta = kind, float(theta)
        self.eps_rho, self.eps_p = float(eps_rho), float(eps_p)
        self.gpu_hooks = {"extrapolate_interface": (
            ("traces_toward_mean", (self.theta,)) if kind == "toward_mean"
            else ("traces_positivity_zhang_shu", (self.eps_rho, self.eps_p)))}

    def element_traces(self, ue, w, lL, lR, gamma=1.4):
        """Host restatement for one element: ue[j, c] (1D Euler, conserved),
        quadrature weights w and Lagrange rows lL, lR -> (trace at xi = -1,
        trace at xi = +1)."""
        import numpy as np

        ue, w = np.asarray(ue, dtype=np.float64), np.asarray(w, dtype=np.float64)
        m = (w @ ue) / w.sum()
        tl, tr = np.asarray(lL) @ ue, np.asarray(lR) @ ue
        if self.kind == "toward_mean":
            return m + self.theta * (tl - m), m + self.theta * (tr - m)
        g1 = gamma - 1.0

        def pres(U):
            return g1 * (U[2] - 0.5 * U[1] * U[1] / U[0])

        if not (m[0] > self.eps_rho) or not (pres(m) > self.eps_p):
            return tl, tr
        rmin = min(tl[0], tr[0])
        if rmin < self.eps_rho:
            th = (m[0] - self.eps_rho) / (m[0] - rmin)
            tl[0], tr[0] = m[0] + th * (tl[0] - m[0]), m[0] + th * (tr[0] - m[0])
        theta = 1.0
        for U in (tl, tr):
            if pres(U) >= self.eps_p:
                continue
            d = U - m
            a = g1 * (d[2] * d[0] - 0.5 * d[1] * d[1])
            b = g1 * (m[2] * d[0] + m[0] * d[2] - m[1] * d[1]) - self.eps_p * d[0]
            c = m[0] * (pres(m) - self.eps_p)
            theta = min(theta, _root01(a, b, c))
        if theta < 1.0:
            tl, tr = m + theta * (tl - m), m + theta * (tr - m)
        return tl, tr

    def extrapolate_interface_(self, traces, u_work, state, eq):
        """Host restatement over a 1D state: traces = (uL[e, c], uR[e, c])."""
        uL, uR = traces
        ops = state.ops
        for e in range(u_work.shape[1]):
            uL[e], uR[e] = self.element_traces(u_work[:, e, :], ops.w, ops.l_L, ops.l_R, eq.gamma)
        return traces

    def method_params(self):
        p = super().method_params()
        p.update({"method": "persson_av_trace_override", "kind": self.kind, "theta": self.theta,
                  "eps_rho": self.eps_rho, "eps_p": self.eps_p})
        return p


_GPU_CLASSES = (ScaledPerssonMethod, PerssonAVMethod, NullCapturing)

# Method registry (Interfaces.jl:118-135, src/methods/Registry.jl:14-53)
METHOD_REGISTRY: Dict[str, Callable[..., AbstractCapturingMethod]] = {
    "null": lambda **kw: NullCapturing(),
    "persson_av": lambda **kw: PerssonAVMethod(**kw),
    "scaled_persson": lambda **kw: ScaledPerssonMethod(**kw),
    "persson_av_positive": lambda **kw: PositivityPreservingPersson(**kw),
    "persson_av_flux_override": lambda **kw: FluxOverridePersson(**kw),
    "persson_av_preprocess_positive": lambda **kw: PositivityPreprocessPersson(**kw),
    "persson_av_trace_override": lambda **kw: TraceOverridePersson(**kw),
}


def register_method(name: str, factory: Callable[..., AbstractCapturingMethod]) -> None:
    METHOD_REGISTRY[str(name)] = factory


def get_capturing_method(name: str, **kwargs) -> AbstractCapturingMethod:
    if name not in METHOD_REGISTRY:
        raise KeyError(f'Unknown capturing method "{name}". Known: {", ".join(sorted(METHOD_REGISTRY))}')
    return METHOD_REGISTRY[name](**kwargs)


def list_methods():
    return sorted(METHOD_REGISTRY)


def method_params(m) -> dict:
    return m.method_params() if hasattr(m, "method_params") else {}
