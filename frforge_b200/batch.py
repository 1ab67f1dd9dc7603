"""Batched execution: many independent solves advanced together on one GPU.

The reference advances one case at a time: its sweep drivers (robustness
matrix ``src/invent/Robustness.jl:245``, confirm presets
``src/invent/Confirm.jl:35-57``, the case runners of ``src/cli/run.jl``) call
``integrate!`` (``src/time/Integrate.jl:9``) once per case.  ``Batch`` runs
such a set of cases as one device job (``frg_batch_*`` in
``include/frforge_cuda.h``): each instance keeps its own mesh, degree, flux,
scheme, dt, time and status, and its result is the one ``integrate_`` gives
for that case alone.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional

import numpy as np

from . import _lib as L
from .gpu import Context, default_context, diagnostics_of, make_desc, set_solve_hooks
from .methods import AbstractCapturingMethod


def solve_bytes(state, eq, method: Optional[AbstractCapturingMethod] = None,
                time: Optional[str] = None) -> int:
    """Upper bound of the device bytes a solve of this state holds."""
    d, _keep = make_desc(state, eq, method, time)
    n = C.c_size_t()
    L.check(L.load().frg_solve_bytes(C.byref(d), C.byref(n)), None, "frg_solve_bytes")
    return int(n.value)


class Batch:
    """A set of instance slots advanced together (``frg_batch``)."""

    def __init__(self, capacity: int, hbm_budget: int = 0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.capacity = int(capacity)
        h = C.c_void_p()
        L.check(L.load().frg_batch_create(self.ctx.handle, self.capacity, int(hbm_budget), C.byref(h)),
                self.ctx.handle, "frg_batch_create")
        self.handle = h
        self._shape: Dict[int, tuple] = {}
        self._ndof: Dict[int, int] = {}
        self._results = (L.frg_result * self.capacity)()

    def close(self):
        if getattr(self, "handle", None):
            L.load().frg_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, code, what):
        return L.check(code, self.ctx.handle, what)

    def set_multirate(self, on: bool = True) -> None:
        """Multirate scheduling: groups with cheaper steps take more steps per
        round (results are unchanged; ``run``'s max_steps counts rounds)."""
        self._chk(L.load().frg_batch_set_multirate(self.handle, 1 if on else 0), "frg_batch_set_multirate")

    def group_of(self, slot: int):
        """(tile variant, solo) of the group the slot ran in at the last run:
        the autotune table's variant for its key, or -1 for the default tile."""
        v, s = C.c_int(), C.c_int()
        self._chk(L.load().frg_batch_slot_group(self.handle, int(slot), C.byref(v), C.byref(s)),
                  "frg_batch_slot_group")
        return v.value, bool(s.value)

    def _solve(self, slot: int):
        s = C.c_void_p()
        self._chk(L.load().frg_batch_get_solve(self.handle, int(slot), C.byref(s)), "frg_batch_get_solve")
        return s

    def hook_calls(self, slot: int) -> dict:
        """Device-counted hook invocations of the slot's instance (see
        GpuSolve.hook_calls)."""
        c = (C.c_int64 * len(L.HOOK_SLOT))()
        self._chk(L.load().frg_solve_hook_calls(self._solve(slot), c, len(c)), "frg_solve_hook_calls")
        return {name: (None if c[i] < 0 else int(c[i])) for name, i in L.HOOK_SLOT.items()}

    def add(self, state, eq, method: Optional[AbstractCapturingMethod] = None, time: Optional[str] = None,
            caller_ops=None) -> int:
        """Create an instance for ``state`` (its u and t are uploaded); returns
        its slot.  Raises FRGError (FRG_ERR_OOM) when the batch is full or its
        HBM budget would be exceeded.  The device hooks the method selects
        (post_step) run on the instance after each of its completed steps."""
        d, _keep = make_desc(state, eq, method, time, caller_ops)
        slot = C.c_int()
        self._chk(L.load().frg_batch_add(self.handle, C.byref(d), C.byref(slot)), "frg_batch_add")
        i = slot.value
        try:
            set_solve_hooks(self._solve(i), self.ctx, method)
        except Exception:
            self.remove(i)
            raise
        self._shape[i] = state.u.shape
        self._ndof[i] = int(state.u.size)
        self.upload(i, state.u, state.t)
        return i

    def remove(self, slot: int) -> None:
        self._chk(L.load().frg_batch_remove(self.handle, int(slot)), "frg_batch_remove")
        self._shape.pop(slot, None)
        self._ndof.pop(slot, None)

    def upload(self, slot: int, u: np.ndarray, t: float) -> None:
        flat = np.ascontiguousarray(np.asarray(u, dtype=np.float64).ravel(order="F"))
        self._chk(L.load().frg_upload_state(self._solve(slot), L.dptr(flat), flat.size, float(t)),
                  "upload")

    def upload_ptr(self, slot: int, host_ptr: int, t: float) -> None:
        self._chk(L.load().frg_upload_state(self._solve(slot), C.cast(host_ptr, L._dp), self._ndof[slot],
                                            float(t)), "upload")

    def download(self, slot: int):
        flat = np.empty(self._ndof[slot])
        t = C.c_double()
        self._chk(L.load().frg_download_state(self._solve(slot), L.dptr(flat), flat.size, C.byref(t)),
                  "download")
        return flat.reshape(self._shape[slot], order="F"), t.value

    def download_ptr(self, slot: int, host_ptr: int) -> float:
        t = C.c_double()
        self._chk(L.load().frg_download_state(self._solve(slot), C.cast(host_ptr, L._dp), self._ndof[slot],
                                              C.byref(t)), "download")
        return t.value

    def set_initial_condition(self, slot: int, kind: str, prim=(), x0: float = 0.5, y0: float = 0.5,
                              amp: float = 0.0, phase: float = 0.0, t: float = 0.0) -> None:
        """Evaluate a case IC on the device into the instance's state (time 0)."""
        ic = L.make_ic(kind, prim, x0, y0, amp, phase, t)
        self._chk(L.load().frg_set_initial_condition(self._solve(slot), C.byref(ic)), "frg_set_initial_condition")

    def diagnostics(self, slot: int, exact: str = "none", t_exact: float = 0.0, c: int = 0) -> dict:
        """Device-side scoring reductions of an instance's state (see
        GpuSolve.diagnostics)."""
        neq = 4 if len(self._shape[slot]) == 4 else 3
        return diagnostics_of(self._solve(slot), self.ctx, exact, t_exact, c, 0, neq)

    def start(self, slot: int, t_final: float, cfl: float = 0.2, dt: Optional[float] = None,
              max_steps: int = 10**7) -> None:
        """Start the instance's run with integrate_'s arguments."""
        self._chk(L.load().frg_batch_start(self.handle, int(slot), float(t_final), float(cfl),
                                           -1.0 if dt is None else float(dt), int(max_steps)),
                  "frg_batch_start")

    def run(self, max_steps: int = 2**62) -> List[Optional[dict]]:
        """Advance the running instances by up to ``max_steps`` steps (or until
        none runs); returns per slot None (empty) or {status, n_steps, t}."""
        n = C.c_int()
        self._chk(L.load().frg_batch_run(self.handle, int(max_steps), self._results, C.byref(n)),
                  "frg_batch_run")
        self.n_running = n.value
        out: List[Optional[dict]] = []
        for i in range(self.capacity):
            r = self._results[i]
            if r.status == L.FRG_ERR_STATE:
                out.append(None)
            else:
                out.append({"status": L.STATUS_SYMBOL[r.status], "n_steps": int(r.n_steps), "t": r.t})
        return out
