"""GPU execution of the FR residual + SSP-RK path through the C ABI.

These functions are the drop-in counterparts of the reference's
``residual!`` (src/fr/Residual.jl:161, Residual2D.jl:131), ``sense!``,
``compute_dt`` (src/time/SSP_RK3.jl:8, :126), ``ssp_rk3_step!`` /
``ssp_rk2_step!``, ``ssp_rk3!`` / ``ssp_rk2!`` and ``integrate!``
(src/time/Integrate.jl:9).  Python has no ``!``; a trailing underscore marks
the in-place functions (``residual_``, ``integrate_``).  The host numpy state
stays the source of truth between calls: each call uploads ``state.u``,
runs on the device and writes the result back, like the Julia arrays.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import Optional

import numpy as np

from . import _lib as L
from .methods import AbstractCapturingMethod, NullCapturing
from .mesh import AbstractBC

_ctx_lock = threading.Lock()
_contexts = {}


class Context:
    """One frg_ctx (device + CUDA stream); one per host thread and device."""

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        L.check(L.load().frg_ctx_create(device, C.byref(h)), what=f"frg_ctx_create(device={device})")
        self.handle = h

    def close(self):
        if self.handle:
            L.load().frg_ctx_destroy(self.handle)
            self.handle = None

    def stream_handle(self) -> int:
        """cudaStream_t of this context (wrap with torch.cuda.ExternalStream)."""
        st = C.c_void_p()
        L.check(L.load().frg_ctx_get_stream(self.handle, C.byref(st)), what="frg_ctx_get_stream")
        return st.value or 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context(device: int = 0) -> Context:
    key = (threading.get_ident(), device)
    with _ctx_lock:
        if key not in _contexts:
            _contexts[key] = Context(device)
        return _contexts[key]


def _bc_struct(bc: AbstractBC) -> L.frg_bc:
    b = L.frg_bc()
    b.kind = L.BC_KIND[bc.kind]
    b.sdiv = 1.0
    if bc.kind == "dirichlet":
        st = np.asarray(bc.state, dtype=np.float64).ravel()
        for i, v in enumerate(st):
            b.state[i] = v
    elif bc.kind == "xsplit":
        for i, v in enumerate(bc.state):
            b.state[i] = v
        if bc.state_b is not None:
            for i, v in enumerate(bc.state_b):
                b.state_b[i] = v
        b.mode = 0 if bc.right_reflect else 1
        b.x0, b.s0, b.s1, b.sdiv = bc.x0, bc.s0, bc.s1, bc.sdiv
    return b


def make_desc(state, eq, method: Optional[AbstractCapturingMethod] = None, time: Optional[str] = None,
              caller_ops=None):
    """frg_solve_desc of a solution state + method; returns (desc, keep): keep
    holds the host arrays the descriptor points into (alive until the solve is
    created)."""
    method = method or NullCapturing()
    spec = method.gpu_spec()
    d = L.frg_solve_desc()
    keep = []
    sch = state.scheme
    d.dim = state.dim
    d.p = state.ops.p
    d.points = L.POINTS[sch.points]
    d.flux = L.FLUX[sch.flux]
    d.time_scheme = L.TIME[time or sch.time]
    d.gamma = eq.gamma
    m = state.mesh
    xv = np.ascontiguousarray(m.x_vertices)
    keep.append(xv)
    d.x_vertices = L.dptr(xv)
    if state.dim == 1:
        d.nx, d.ny = m.n_elements, 1
        d.x_left, d.x_right = m.x_left, m.x_right
        d.bc[0] = _bc_struct(m.left_bc)
        d.bc[1] = _bc_struct(m.right_bc)
    else:
        d.nx, d.ny = m.nx, m.ny
        d.x_left, d.x_right, d.y_bottom, d.y_top = m.x_left, m.x_right, m.y_bottom, m.y_top
        yv = np.ascontiguousarray(m.y_vertices)
        keep.append(yv)
        d.y_vertices = L.dptr(yv)
        for k, bc in enumerate((m.left_bc, m.right_bc, m.bottom_bc, m.top_bc)):
            d.bc[k] = _bc_struct(bc)
        if m.solid is not None:
            sol = np.ascontiguousarray(m.solid, dtype=np.uint8)
            keep.append(sol)
            d.solid = sol.ctypes.data_as(C.c_void_p)
        if state.metrics is not None:
            mt = L.frg_metrics2d()
            for name in L._METRIC_FIELDS:
                a = np.asfortranarray(state.metrics[name], dtype=np.float64).ravel(order="F")
                a = np.ascontiguousarray(a)
                keep.append(a)
                setattr(mt, name, L.dptr(a))
            keep.append(mt)
            d.geometry = L.GEOM["metrics"]
            d.metrics = C.pointer(mt)
        elif state.wavy_amp is not None:
            d.geometry = L.GEOM["wavy"]
            d.wavy_amp = state.wavy_amp
    if caller_ops is not None:
        o = L.frg_operators()
        o.p = caller_ops["p"] if isinstance(caller_ops, dict) else caller_ops.p
        o.points = d.points
        for name in ("xi", "w", "D", "l_L", "l_R", "gL_xi", "gR_xi", "V"):
            src = caller_ops[name] if isinstance(caller_ops, dict) else getattr(
                caller_ops, "V_legendre" if name == "V" else name)
            a = np.ascontiguousarray(np.asarray(src, dtype=np.float64).ravel(order="F"))
            keep.append(a)
            setattr(o, name, L.dptr(a))
        keep.append(o)
        d.ops = C.pointer(o)
    d.method = L.METHOD[spec["method"]]
    d.av_form = L.AV_FORM[spec["av_form"]]
    d.kappa, d.s0_factor, d.eps_floor, d.c_av = (spec["kappa"], spec["s0_factor"],
                                                spec["eps_floor"], spec["c_av"])
    return d, keep


def diagnostics_of(handle, ctx, exact: str, t_exact: float, c: int, ref_ptr: int, neq: int) -> dict:
    d = L.frg_diagnostics()
    L.check(L.load().frg_diagnostics_compute(handle, L.EXACT[exact], C.c_void_p(ref_ptr or None), float(t_exact),
                                             int(c), C.byref(d)), ctx.handle, "frg_diagnostics_compute")
    return {"mass": [d.mass[k] for k in range(neq)], "rho_min": d.rho_min, "rho_max": d.rho_max,
            "p_min": d.p_min, "nonfinite": int(d.nonfinite), "positivity_ok": bool(d.positivity_ok),
            "l2_error": d.l2_error, "t": d.t}


def method_hooks(method: Optional[AbstractCapturingMethod]):
    """The device hooks a method selects: [(slot id, hook id, params)] from its
    gpu_spec()["hooks"] {slot name: (implementation name, params)}, resolved
    through the registry (frg_hook_lookup)."""
    out = []
    for slot, (name, params) in (method or NullCapturing()).gpu_spec().get("hooks", {}).items():
        sl, hid = C.c_int(), C.c_int()
        L.check(L.load().frg_hook_lookup(name.encode(), C.byref(sl), C.byref(hid)), None, "frg_hook_lookup")
        if sl.value != L.HOOK_SLOT[slot]:
            raise ValueError(f"{name} implements another hook slot")
        out.append((sl.value, hid.value, np.ascontiguousarray(np.asarray(params, dtype=np.float64))))
    return out


def set_solve_hooks(handle, ctx: "Context", method: Optional[AbstractCapturingMethod]) -> None:
    """Select on solve `handle` the device hooks of `method` (frg_solve_set_hook)."""
    for sl, hid, arr in method_hooks(method):
        L.check(L.load().frg_solve_set_hook(handle, sl, hid, L.dptr(arr) if arr.size else None, int(arr.size)),
                ctx.handle, "frg_solve_set_hook")


class GpuSolve:
    """A device-resident solve (frg_solve): descriptor, state buffers, graphs."""

    def __init__(self, state, eq, method: Optional[AbstractCapturingMethod] = None,
                 time: Optional[str] = None, ctx: Optional[Context] = None, caller_ops=None):
        self.ctx = ctx or default_context()
        self.state_shape = state.u.shape
        d, self._keep = make_desc(state, eq, method, time, caller_ops)
        self.desc = d
        h = C.c_void_p()
        L.check(L.load().frg_solve_create(self.ctx.handle, C.byref(d), C.byref(h)), self.ctx.handle,
                "frg_solve_create")
        self.handle = h
        info = self.info()
        self.ndof, self.nel = info["ndof"], info["nel"]
        # device implementations of the hooks the method overrides
        set_solve_hooks(self.handle, self.ctx, method)

    def set_hook(self, slot: str, name: str, params=()) -> None:
        """Select the device implementation `name` of hook `slot`
        ("post_step"); see frg_solve_set_hook."""
        sl, hid = C.c_int(), C.c_int()
        self._chk(L.load().frg_hook_lookup(name.encode(), C.byref(sl), C.byref(hid)), "frg_hook_lookup")
        if sl.value != L.HOOK_SLOT[slot]:
            raise ValueError(f"{name} implements another hook slot")
        arr = np.ascontiguousarray(np.asarray(params, dtype=np.float64))
        self._chk(L.load().frg_solve_set_hook(self.handle, sl.value, hid.value, L.dptr(arr) if arr.size else None,
                                              int(arr.size)), "frg_solve_set_hook")

    def apply_post_step(self) -> None:
        """Run the post-step hook once on the current state."""
        self._chk(L.load().frg_apply_post_step(self.handle), "frg_apply_post_step")

    def hook_calls(self) -> dict:
        """Device-counted invocations per hook slot since the solve was made
        (the HookProbeMethod counters of test/test_capturing.jl); the inline
        numerical_flux_method and extrapolate_interface slots report None."""
        c = (C.c_int64 * len(L.HOOK_SLOT))()
        self._chk(L.load().frg_solve_hook_calls(self.handle, c, len(c)), "frg_solve_hook_calls")
        return {name: (None if c[i] < 0 else int(c[i])) for name, i in L.HOOK_SLOT.items()}

    def close(self):
        if getattr(self, "handle", None):
            L.load().frg_solve_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, code, what):
        return L.check(code, self.ctx.handle, what)

    def info(self) -> dict:
        i = L.frg_solve_info()
        self._chk(L.load().frg_solve_get_info(self.handle, C.byref(i)), "frg_solve_get_info")
        return {"ndof": i.ndof, "nel": i.nel, "np": i.np, "neq": i.neq, "device_bytes": i.device_bytes,
                "residual_evals": i.residual_evals, "steps": i.steps}

    def upload(self, u: np.ndarray, t: float) -> None:
        flat = np.ascontiguousarray(np.asarray(u, dtype=np.float64).ravel(order="F"))
        self._chk(L.load().frg_upload_state(self.handle, L.dptr(flat), flat.size, float(t)), "upload")

    def upload_ptr(self, host_ptr: int, t: float) -> None:
        """Upload ndof doubles from a raw host address (e.g. pinned memory)."""
        self._chk(L.load().frg_upload_state(self.handle, C.cast(host_ptr, L._dp), self.ndof, float(t)),
                  "upload")

    def download_ptr(self, host_ptr: int) -> float:
        """Download the state to a raw host address; returns its time."""
        t = C.c_double()
        self._chk(L.load().frg_download_state(self.handle, C.cast(host_ptr, L._dp), self.ndof,
                                              C.byref(t)), "download")
        return t.value

    def download(self):
        flat = np.empty(self.ndof)
        t = C.c_double()
        self._chk(L.load().frg_download_state(self.handle, L.dptr(flat), flat.size, C.byref(t)), "download")
        return flat.reshape(self.state_shape, order="F"), t.value

    def residual(self) -> np.ndarray:
        du = np.empty(self.ndof)
        self._chk(L.load().frg_residual(self.handle, L.dptr(du), du.size), "frg_residual")
        return du.reshape(self.state_shape, order="F")

    def sense(self) -> np.ndarray:
        s = np.empty(self.nel)
        self._chk(L.load().frg_sense(self.handle, L.dptr(s), s.size), "frg_sense")
        return s

    def compute_dt(self, cfl: float) -> float:
        dt = C.c_double()
        self._chk(L.load().frg_compute_dt(self.handle, float(cfl), C.byref(dt)), "frg_compute_dt")
        return dt.value

    def step(self, dt: float) -> str:
        st = C.c_int()
        self._chk(L.load().frg_step(self.handle, float(dt), C.byref(st)), "frg_step")
        return L.STATUS_SYMBOL[st.value]

    def advance(self, t_final: float, cfl: float = 0.2, dt: Optional[float] = None,
                max_steps: int = 10**7) -> dict:
        r = L.frg_result()
        self._chk(L.load().frg_advance(self.handle, float(t_final), float(cfl),
                                       -1.0 if dt is None else float(dt), int(max_steps), C.byref(r)),
                  "frg_advance")
        return {"status": L.STATUS_SYMBOL[r.status], "n_steps": int(r.n_steps), "t": r.t}

    def set_initial_condition(self, kind: str, prim=(), x0: float = 0.5, y0: float = 0.5, amp: float = 0.0,
                              phase: float = 0.0, t: float = 0.0) -> None:
        """set_initial_condition! for a case IC, evaluated on the device
        (see frg_ic in include/frforge_cuda.h); the state time becomes 0."""
        ic = L.make_ic(kind, prim, x0, y0, amp, phase, t)
        self._chk(L.load().frg_set_initial_condition(self.handle, C.byref(ic)), "frg_set_initial_condition")

    def diagnostics(self, exact: str = "none", t_exact: float = 0.0, c: int = 0, ref_ptr: int = 0) -> dict:
        """Device-side scoring reductions of the current state (mass per
        component, density extrema, minimum pressure, non-finite count,
        positivity, and the L2 error of component c against an exact
        solution: "vortex_2d", "smooth_2d", "density_wave_1d", or "state"
        with a device pointer ref_ptr)."""
        return diagnostics_of(self.handle, self.ctx, exact, t_exact, c, ref_ptr, self.info()["neq"])

    def shock_metrics(self, ref=None, ref_min: float = 0.125, ref_max: float = 1.0, grad_frac: float = 0.15,
                      exclude=(), window_sp: int = 30) -> dict:
        """1D shock-capturing scores of the current density on the device
        (Metrics.jl: shock_thickness_sp, overshoot_metric, excess_dissipation
        over smooth_region_mask, and the relative L1): ref is None, a density
        array in x order (e.g. an exact solution at the solution points), or
        another 1D GpuSolve on the same mesh (e.g. the NullCapturing run)."""
        prm = L.frg_shock_params()
        prm.ref_min, prm.ref_max, prm.grad_frac = float(ref_min), float(ref_max), float(grad_frac)
        prm.window_sp = int(window_sp)
        exclude = list(exclude)
        if len(exclude) > 4:
            raise ValueError("at most 4 excluded windows")
        prm.n_exclude = len(exclude)
        for k, (a, b) in enumerate(exclude):
            prm.exclude[k][0], prm.exclude[k][1] = float(a), float(b)
        out = L.frg_shock_metrics()
        ref_arr, ref_solve = None, None
        if isinstance(ref, GpuSolve):
            ref_solve = ref.handle
        elif ref is not None:
            ref_arr = np.ascontiguousarray(np.asarray(ref, dtype=np.float64).ravel())
            if ref_arr.size != self.nel * self.state_shape[0]:
                raise ValueError("reference density must have one value per solution point")
        self._chk(L.load().frg_shock_metrics_1d(self.handle, C.byref(prm),
                                                L.dptr(ref_arr) if ref_arr is not None else None, ref_solve,
                                                C.byref(out)), "frg_shock_metrics_1d")
        has_ref = bool(out.has_reference)
        return {"shock_thickness": out.shock_thickness, "shock_index": int(out.shock_index),
                "shock_x": out.shock_x, "overshoot": out.overshoot, "overshoot_over": out.overshoot_over,
                "overshoot_under": out.overshoot_under, "rho_min": out.rho_min, "rho_max": out.rho_max,
                "excess_dissipation": out.excess_dissipation if has_ref else None,
                "l1_rel": out.l1_rel if has_ref else None, "n_samples": int(out.n_samples)}

    def variant(self):
        """(current tile variant, number of variants) of the stage kernel."""
        v, n = C.c_int(), C.c_int()
        self._chk(L.load().frg_get_variant(self.handle, C.byref(v), C.byref(n)), "frg_get_variant")
        return v.value, n.value

    def set_variant(self, v: int) -> None:
        self._chk(L.load().frg_set_variant(self.handle, int(v)), "frg_set_variant")

    def autotune(self, reps: int = 5):
        """Time every tile variant on the current state and keep the fastest;
        returns (best, per-variant ms)."""
        _, n = self.variant()
        ms = np.zeros(max(n, 1))
        best = C.c_int()
        self._chk(L.load().frg_autotune(self.handle, int(reps), C.byref(best), L.dptr(ms)), "frg_autotune")
        return best.value, ms[:n]

    def time_stages(self, nsteps: int, cfl: float = 0.2, dt: Optional[float] = None):
        """Run nsteps steps with every stage kernel bracketed by CUDA events;
        returns (mean stage-kernel ms per stage, result dict)."""
        ms = np.zeros(3)
        r = L.frg_result()
        self._chk(L.load().frg_time_stages(self.handle, int(nsteps), float(cfl),
                                           -1.0 if dt is None else float(dt), L.dptr(ms), C.byref(r)),
                  "frg_time_stages")
        return ms, {"status": L.STATUS_SYMBOL[r.status], "n_steps": int(r.n_steps), "t": r.t}


def _solve_for(state, eq, method, time=None) -> GpuSolve:
    method = method or NullCapturing()
    spec = method.gpu_spec()
    hooks = tuple(sorted(spec.pop("hooks", {}).items()))
    key = (tuple(sorted(spec.items())), hooks, time or state.scheme.time, state.scheme, eq.gamma)
    s = state._gpu.get(key)
    if s is None:
        s = GpuSolve(state, eq, method, time=time)
        state._gpu[key] = s
    return s


def residual_(du, state, eq, method: Optional[AbstractCapturingMethod] = None):
    """residual!(du, state, eq, method) on the GPU."""
    s = _solve_for(state, eq, method)
    s.upload(state.u, state.t)
    du[...] = s.residual()
    return du


def sense_(sigma, method, state, eq):
    """sense!(sigma, method, u_work, state, eq): Persson element sensor."""
    s = _solve_for(state, eq, method)
    s.upload(state.u, state.t)
    sigma[...] = s.sense()
    return sigma


def compute_dt(state, eq, cfl: float = 0.2) -> float:
    s = _solve_for(state, eq, None)
    s.upload(state.u, state.t)
    return s.compute_dt(cfl)


def _step(state, eq, method, dt, time):
    s = _solve_for(state, eq, method, time)
    s.upload(state.u, state.t)
    status = s.step(dt)
    state.u[...], state.t = s.download()
    return status


def ssp_rk3_step_(state, eq, method, dt: float) -> str:
    """ssp_rk3_step! (SSP_RK3.jl:29-65, :135-164): 'ok' or 'diverged'."""
    return _step(state, eq, method, dt, "ssp_rk3")


def ssp_rk2_step_(state, eq, method, dt: float) -> str:
    """ssp_rk2_step! (SSP_RK2.jl:14-68)."""
    return _step(state, eq, method, dt, "ssp_rk2")


def _run(state, eq, method, t_final, cfl, dt, max_steps, time):
    s = _solve_for(state, eq, method, time)
    s.upload(state.u, state.t)
    r = s.advance(t_final, cfl=cfl, dt=dt, max_steps=max_steps)
    state.u[...], state.t = s.download()
    return r


def ssp_rk3_(state, eq, method, t_final, cfl=0.2, dt=None, max_steps=10**7) -> dict:
    """ssp_rk3!(state, eq, method, t_final; cfl, dt, max_steps)."""
    return _run(state, eq, method, t_final, cfl, dt, max_steps, "ssp_rk3")


def ssp_rk2_(state, eq, method, t_final, cfl=0.2, dt=None, max_steps=10**7) -> dict:
    return _run(state, eq, method, t_final, cfl, dt, max_steps, "ssp_rk2")


def integrate_(state, eq, method, t_final, cfl=0.2, dt=None, max_steps=10**7, time=None) -> dict:
    """integrate!(state, eq, method, t_final; cfl, dt, max_steps, time)
    (src/time/Integrate.jl:9-43)."""
    tsym = time or state.scheme.time
    if tsym not in ("ssp_rk3", "ssp_rk2"):
        raise ValueError(f"Unknown time scheme {tsym} (use :ssp_rk3 or :ssp_rk2)")
    return _run(state, eq, method, t_final, cfl, dt, max_steps, tsym)
