"""Served execution: a request queue in front of a batch (``frg_server_*``).

The reference serves one case at a time (its case runners, e.g.
``src/cli/run.jl:267``, call ``integrate!`` per request).  ``Server`` queues
requests, admits them in arrival order into free batch slots while their
device footprint fits the HBM budget, advances the batch in bounded pumps and
delivers each finished request's state and status.  A request's result is the
one it gets alone in a batch, whatever else is being served.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional

import numpy as np

from . import _lib as L
from .gpu import Context, default_context, make_desc, method_hooks
from .methods import AbstractCapturingMethod


class Server:
    """``frg_server``: ``slots`` concurrent solves, ``steps_per_pump`` rounds
    per pump, multirate scheduling."""

    def __init__(self, slots: int = 64, hbm_budget: int = 0, steps_per_pump: int = 16,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        L.check(L.load().frg_server_create(self.ctx.handle, int(slots), int(hbm_budget), int(steps_per_pump),
                                           C.byref(h)), self.ctx.handle, "frg_server_create")
        self.handle = h
        self._req: Dict[int, tuple] = {}

    def close(self):
        if getattr(self, "handle", None):
            L.load().frg_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, code, what):
        return L.check(code, self.ctx.handle, what)

    def submit(self, state, eq, method: Optional[AbstractCapturingMethod] = None, t_final: float = 1.0,
               cfl: float = 0.2, dt: Optional[float] = None, max_steps: int = 10**7,
               time: Optional[str] = None, want_state: bool = True) -> int:
        """Queue ``integrate_(state, eq, method, t_final; cfl, dt, max_steps)``;
        returns the request id.  want_state=False: only the device-side
        diagnostics of the final state are returned, not the state."""
        d, keep = make_desc(state, eq, method, time)
        hooks = method_hooks(method)
        u0 = np.ascontiguousarray(np.asarray(state.u, dtype=np.float64).ravel(order="F"))
        out = np.empty_like(u0) if want_state else None
        rid = C.c_int64()
        self._chk(L.load().frg_server_submit(self.handle, C.byref(d), L.dptr(u0), float(state.t), float(t_final),
                                             float(cfl), -1.0 if dt is None else float(dt), int(max_steps),
                                             L.dptr(out) if want_state else None, C.byref(rid)),
                  "frg_server_submit")
        self._req[rid.value] = (d, keep, u0, out, state.u.shape)
        self._set_hooks(rid.value, hooks)
        return rid.value

    def submit_ic(self, state, eq, ic: dict, method: Optional[AbstractCapturingMethod] = None,
                  t_final: float = 1.0, cfl: float = 0.2, dt: Optional[float] = None, max_steps: int = 10**7,
                  time: Optional[str] = None, want_state: bool = True) -> int:
        """As submit, with the initial state evaluated on the device at
        admission from the case IC ``ic`` (keyword arguments of
        frforge_b200._lib.make_ic); ``state`` gives the mesh and scheme only."""
        d, keep = make_desc(state, eq, method, time)
        hooks = method_hooks(method)
        c_ic = L.make_ic(**ic)
        out = np.empty(int(np.prod(state.u.shape))) if want_state else None
        rid = C.c_int64()
        self._chk(L.load().frg_server_submit_ic(self.handle, C.byref(d), C.byref(c_ic), float(t_final), float(cfl),
                                                -1.0 if dt is None else float(dt), int(max_steps),
                                                L.dptr(out) if want_state else None, C.byref(rid)),
                  "frg_server_submit_ic")
        self._req[rid.value] = (d, keep, None, out, state.u.shape)
        self._set_hooks(rid.value, hooks)
        return rid.value

    def _set_hooks(self, rid: int, hooks) -> None:
        """Attach the method's device hooks to the queued request (applied at
        admission, frg_server_set_hook); a refused hook cancels the request."""
        for sl, hid, arr in hooks:
            code = L.load().frg_server_set_hook(self.handle, int(rid), sl, hid, L.dptr(arr) if arr.size else None,
                                                int(arr.size))
            if code:
                L.load().frg_server_cancel(self.handle, int(rid))
                self._chk(code, "frg_server_set_hook")

    def cancel(self, rid: int) -> None:
        self._chk(L.load().frg_server_cancel(self.handle, int(rid)), "frg_server_cancel")

    def pump(self):
        """One scheduling round: (completed by this call, queued, running)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._chk(L.load().frg_server_pump(self.handle, C.byref(a), C.byref(b), C.byref(c)), "frg_server_pump")
        return a.value, b.value, c.value

    def take_completed(self) -> List[int]:
        ids = (C.c_int64 * 256)()
        out: List[int] = []
        while True:
            n = C.c_int()
            self._chk(L.load().frg_server_take_completed(self.handle, ids, 256, C.byref(n)),
                      "frg_server_take_completed")
            out.extend(ids[k] for k in range(n.value))
            if n.value < 256:
                return out

    def result(self, rid: int, release: bool = True) -> Optional[dict]:
        """{status, n_steps, t, u} once the request completed, else None."""
        done = C.c_int()
        r = L.frg_result()
        self._chk(L.load().frg_server_result(self.handle, int(rid), C.byref(done), C.byref(r)),
                  "frg_server_result")
        if not done.value:
            return None
        d, keep, u0, out, shape = self._req[rid]
        if release:
            del self._req[rid]
        st = r.status
        res = {"status": L.STATUS_SYMBOL.get(st, st), "n_steps": int(r.n_steps), "t": r.t,
               "u": out.reshape(shape, order="F") if out is not None else None, "diagnostics": None}
        dg = L.frg_diagnostics()
        if L.load().frg_server_diagnostics(self.handle, int(rid), C.byref(dg)) == L.FRG_OK:
            neq = 4 if len(shape) == 4 else 3
            res["diagnostics"] = {"mass": [dg.mass[k] for k in range(neq)], "rho_min": dg.rho_min,
                                  "rho_max": dg.rho_max, "p_min": dg.p_min, "nonfinite": int(dg.nonfinite),
                                  "positivity_ok": bool(dg.positivity_ok), "t": dg.t}
        return res

    def drain(self, max_pumps: int = 10**9) -> None:
        """Pump until nothing is queued or running."""
        for _ in range(max_pumps):
            _, q, a = self.pump()
            if q == 0 and a == 0:
                return
