"""ctypes binding of the C ABI declared in include/frforge_cuda.h.

The shared library is built in-tree (``frforge_b200/libfrforge_cuda.so``).
There is no fallback: if the library or a GPU is missing, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfrforge_cuda.so")

# status codes (frg_status)
FRG_OK, FRG_DIVERGED, FRG_MAX_STEPS, FRG_RUNNING, FRG_CANCELLED = 0, 1, 2, 3, 4
FRG_ERR_INVALID_ARG, FRG_ERR_UNSUPPORTED_HOOK, FRG_ERR_OOM = -1, -2, -3
FRG_ERR_CUDA, FRG_ERR_TIMEOUT, FRG_ERR_STATE = -4, -5, -6

POINTS = {"gl": 0, "gll": 1}
FLUX = {"rusanov": 0, "hllc": 1}
TIME = {"ssp_rk3": 0, "ssp_rk2": 1}
BC_KIND = {"periodic": 0, "transmissive": 1, "dirichlet": 2, "reflecting": 3, "xsplit": 4}
METHOD = {"null": 0, "persson": 1}
AV_FORM = {"conservative_br0": 0, "element_local_DD": 1}
GEOM = {"affine": 0, "wavy": 1, "metrics": 2}
STATUS_SYMBOL = {FRG_OK: "ok", FRG_DIVERGED: "diverged", FRG_MAX_STEPS: "max_steps",
                 FRG_RUNNING: "running", FRG_CANCELLED: "cancelled"}

_dp = C.POINTER(C.c_double)


class frg_bc(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("mode", C.c_int),
        ("state", C.c_double * 4), ("state_b", C.c_double * 4),
        ("x0", C.c_double), ("s0", C.c_double), ("s1", C.c_double), ("sdiv", C.c_double),
    ]


class frg_operators(C.Structure):
    _fields_ = [
        ("p", C.c_int), ("points", C.c_int),
        ("xi", _dp), ("w", _dp), ("D", _dp), ("l_L", _dp), ("l_R", _dp),
        ("gL_xi", _dp), ("gR_xi", _dp), ("V", _dp),
    ]


_METRIC_FIELDS = ["x_xi", "x_eta", "y_xi", "y_eta", "J",
                  "nx_W", "ny_W", "sJ_W", "nx_E", "ny_E", "sJ_E",
                  "nx_S", "ny_S", "sJ_S", "nx_N", "ny_N", "sJ_N", "h_char"]


class frg_metrics2d(C.Structure):
    _fields_ = [(n, _dp) for n in _METRIC_FIELDS]


class frg_solve_desc(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("p", C.c_int), ("points", C.c_int), ("flux", C.c_int),
        ("time_scheme", C.c_int), ("gamma", C.c_double),
        ("nx", C.c_int), ("ny", C.c_int),
        ("x_left", C.c_double), ("x_right", C.c_double),
        ("y_bottom", C.c_double), ("y_top", C.c_double),
        ("x_vertices", _dp), ("y_vertices", _dp),
        ("bc", frg_bc * 4),
        ("solid", C.c_void_p),
        ("geometry", C.c_int), ("wavy_amp", C.c_double),
        ("metrics", C.POINTER(frg_metrics2d)),
        ("ops", C.POINTER(frg_operators)),
        ("method", C.c_int), ("av_form", C.c_int),
        ("kappa", C.c_double), ("s0_factor", C.c_double),
        ("eps_floor", C.c_double), ("c_av", C.c_double),
    ]


class frg_result(C.Structure):
    _fields_ = [("status", C.c_int), ("n_steps", C.c_int64), ("t", C.c_double)]


class frg_diagnostics(C.Structure):
    _fields_ = [("mass", C.c_double * 4), ("rho_min", C.c_double), ("rho_max", C.c_double),
                ("p_min", C.c_double), ("nonfinite", C.c_int64), ("positivity_ok", C.c_int),
                ("pad", C.c_int), ("l2_error", C.c_double), ("t", C.c_double)]


class frg_shock_params(C.Structure):
    _fields_ = [("ref_min", C.c_double), ("ref_max", C.c_double), ("grad_frac", C.c_double),
                ("window_sp", C.c_int), ("n_exclude", C.c_int), ("exclude", (C.c_double * 2) * 4)]


class frg_shock_metrics(C.Structure):
    _fields_ = [("shock_thickness", C.c_double), ("shock_index", C.c_int64), ("shock_x", C.c_double),
                ("overshoot", C.c_double), ("overshoot_over", C.c_double), ("overshoot_under", C.c_double),
                ("rho_min", C.c_double), ("rho_max", C.c_double), ("excess_dissipation", C.c_double),
                ("l1_rel", C.c_double), ("n_samples", C.c_int64), ("has_reference", C.c_int),
                ("pad", C.c_int)]


class frg_ic(C.Structure):
    _fields_ = [("kind", C.c_int), ("pad", C.c_int), ("x0", C.c_double), ("y0", C.c_double),
                ("amp", C.c_double), ("phase", C.c_double), ("t", C.c_double), ("prim", (C.c_double * 4) * 4)]


IC_KIND = {"uniform": 0, "two_state": 1, "four_quadrant": 2, "density_wave": 3, "vortex": 4, "smooth_2d": 5,
           "shu_osher": 6}


def make_ic(kind: str, prim=(), x0: float = 0.5, y0: float = 0.5, amp: float = 0.0, phase: float = 0.0,
            t: float = 0.0) -> frg_ic:
    """frg_ic of a case initial condition; prim: up to four primitive states."""
    ic = frg_ic()
    ic.kind = IC_KIND[kind]
    ic.x0, ic.y0, ic.amp, ic.phase, ic.t = float(x0), float(y0), float(amp), float(phase), float(t)
    for r, row in enumerate(prim):
        for c, v in enumerate(row):
            ic.prim[r][c] = float(v)
    return ic


HOOK_SLOT = {"post_step": 0, "numerical_flux_method": 1, "preprocess_state": 2, "extrapolate_interface": 3}


def device_hooks() -> dict:
    """Registered device hook implementations: name -> (slot, id, nparams)."""
    out = {}
    lib = load()
    for i in range(lib.frg_hook_count()):
        name, slot, hid, npar = C.c_char_p(), C.c_int(), C.c_int(), C.c_int()
        lib.frg_hook_info(i, C.byref(name), C.byref(slot), C.byref(hid), C.byref(npar))
        out[name.value.decode()] = (slot.value, hid.value, npar.value)
    return out


EXACT = {"none": 0, "state": 1, "vortex_2d": 2, "smooth_2d": 3, "density_wave_1d": 4}


class frg_solve_info(C.Structure):
    _fields_ = [("ndof", C.c_size_t), ("nel", C.c_int), ("np", C.c_int), ("neq", C.c_int),
                ("device_bytes", C.c_size_t), ("residual_evals", C.c_int64), ("steps", C.c_int64)]


# Every symbol declared in include/frforge_cuda.h with its ctypes signature.
SIGNATURES = {
    "frg_abi_version": (C.c_int, []),
    "frg_version": (C.c_char_p, []),
    "frg_status_string": (C.c_char_p, [C.c_int]),
    "frg_build_operators": (C.c_int, [C.c_int, C.c_int] + [_dp] * 10),
    "frg_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "frg_ctx_destroy": (C.c_int, [C.c_void_p]),
    "frg_last_error": (C.c_char_p, [C.c_void_p]),
    "frg_ctx_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "frg_solve_create": (C.c_int, [C.c_void_p, C.POINTER(frg_solve_desc), C.POINTER(C.c_void_p)]),
    "frg_solve_destroy": (C.c_int, [C.c_void_p]),
    "frg_solve_get_info": (C.c_int, [C.c_void_p, C.POINTER(frg_solve_info)]),
    "frg_upload_state": (C.c_int, [C.c_void_p, _dp, C.c_size_t, C.c_double]),
    "frg_download_state": (C.c_int, [C.c_void_p, _dp, C.c_size_t, C.POINTER(C.c_double)]),
    "frg_residual": (C.c_int, [C.c_void_p, _dp, C.c_size_t]),
    "frg_sense": (C.c_int, [C.c_void_p, _dp, C.c_size_t]),
    "frg_compute_dt": (C.c_int, [C.c_void_p, C.c_double, _dp]),
    "frg_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
    "frg_advance": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int64,
                              C.POINTER(frg_result)]),
    "frg_time_stages": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double, _dp,
                                  C.POINTER(frg_result)]),
    "frg_get_variant": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "frg_set_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "frg_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), _dp]),
    "frg_autotune_table_load": (C.c_int, [C.c_char_p]),
    "frg_autotune_table_save": (C.c_int, [C.c_char_p]),
    "frg_autotune_table_set": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "frg_autotune_table_get": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "frg_autotune_table_clear": (C.c_int, []),
    "frg_autotune_table_size": (C.c_int, []),
    "frg_residual2d_noalloc": (C.c_int, [C.POINTER(frg_solve_desc), C.c_void_p, C.c_void_p,
                                         C.c_double, C.c_void_p]),
    "frg_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
    "frg_batch_destroy": (C.c_int, [C.c_void_p]),
    "frg_batch_add": (C.c_int, [C.c_void_p, C.POINTER(frg_solve_desc), C.POINTER(C.c_int)]),
    "frg_batch_remove": (C.c_int, [C.c_void_p, C.c_int]),
    "frg_batch_get_solve": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "frg_batch_slot_group": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "frg_batch_set_multirate": (C.c_int, [C.c_void_p, C.c_int]),
    "frg_batch_start": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_int64]),
    "frg_batch_run": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(frg_result), C.POINTER(C.c_int)]),
    "frg_solve_bytes": (C.c_int, [C.POINTER(frg_solve_desc), C.POINTER(C.c_size_t)]),
    "frg_set_initial_condition": (C.c_int, [C.c_void_p, C.POINTER(frg_ic)]),
    "frg_hook_count": (C.c_int, []),
    "frg_hook_info": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_int)]),
    "frg_hook_lookup": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "frg_solve_set_hook": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int]),
    "frg_apply_post_step": (C.c_int, [C.c_void_p]),
    "frg_solve_hook_calls": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.c_int]),
    "frg_server_set_hook": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_int, _dp, C.c_int]),
    "frg_server_submit_ic": (C.c_int, [C.c_void_p, C.POINTER(frg_solve_desc), C.POINTER(frg_ic), C.c_double,
                                       C.c_double, C.c_double, C.c_int64, _dp, C.POINTER(C.c_int64)]),
    "frg_vtk_point_data": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, C.c_size_t]),
    "frg_diagnostics_compute": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_int,
                                          C.POINTER(frg_diagnostics)]),
    "frg_server_create": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.c_int64, C.POINTER(C.c_void_p)]),
    "frg_server_destroy": (C.c_int, [C.c_void_p]),
    "frg_server_submit": (C.c_int, [C.c_void_p, C.POINTER(frg_solve_desc), _dp, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_int64, _dp, C.POINTER(C.c_int64)]),
    "frg_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
    "frg_server_pump": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "frg_server_result": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int), C.POINTER(frg_result)]),
    "frg_server_take_completed": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.c_int,
                                            C.POINTER(C.c_int)]),
    "frg_server_diagnostics": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(frg_diagnostics)]),
    "frg_shock_metrics_1d": (C.c_int, [C.c_void_p, C.POINTER(frg_shock_params), _dp, C.c_void_p,
                                       C.POINTER(frg_shock_metrics)]),
}

_lib = None


class FRGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (frg status {code})")
        self.code = code


class UnsupportedHookError(FRGError):
    """A capturing method overrides a hook that has no GPU implementation."""


def load():
    """Load libfrforge_cuda.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m frforge_b200.build` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(code: int, ctx=None, what: str = "") -> int:
    if code < 0:
        msg = what
        if ctx:
            err = load().frg_last_error(ctx)
            if err:
                msg = f"{what}: {err.decode()}"
        if code == FRG_ERR_UNSUPPORTED_HOOK:
            raise UnsupportedHookError(code, msg)
        if code == FRG_ERR_INVALID_ARG:
            raise ValueError(msg)
        raise FRGError(code, msg)
    return code


def dptr(a):
    return a.ctypes.data_as(_dp)
