"""The extrapolate_interface slot's host side (no GPU): the registry resolves
the plugin's device implementations to that slot, the plugin's descriptor
names them, an override without a device name is refused, and the plugin's
host restatement of the traces equals the oracle's (the traces its last
residual's interface fluxes used) element by element."""
import ctypes as C

import numpy as np
import pytest

import frforge_b200 as F
import oracle as O
from frforge_b200 import _lib as L


@pytest.mark.parametrize("name", ["traces_toward_mean", "traces_positivity_zhang_shu"])
def test_registry_resolves_to_the_trace_slot(name):
    sl, hid = C.c_int(), C.c_int()
    assert L.load().frg_hook_lookup(name.encode(), C.byref(sl), C.byref(hid)) == 0
    assert sl.value == L.HOOK_SLOT["extrapolate_interface"] and hid.value > 0


def test_plugin_descriptor_names_the_device_hook():
    spec = F.TraceOverridePersson("toward_mean", theta=0.4, c_av=0.2).gpu_spec()
    assert spec["method"] == "persson" and spec["c_av"] == 0.2
    assert spec["hooks"] == {"extrapolate_interface": ("traces_toward_mean", (0.4,))}
    m = F.get_capturing_method("persson_av_trace_override", kind="positivity", eps_rho=0.01, eps_p=0.02)
    assert m.gpu_spec()["hooks"] == {"extrapolate_interface": ("traces_positivity_zhang_shu", (0.01, 0.02))}


def test_an_override_without_a_device_name_is_refused():
    class HostOnlyTraces(F.PerssonAVMethod):
        def extrapolate_interface_(self, traces, u_work, state, eq):
            return traces

    with pytest.raises(L.UnsupportedHookError):
        HostOnlyTraces().gpu_spec()


def _spoiled_wave(orc):
    orc.ic_density_wave()
    u = orc.u.copy()
    u[0, 3, 0] = 0.02   # end-point densities that push the Lagrange traces below zero
    u[3, 8, 0] = 0.01
    u[1, 14, 2] *= 0.05  # and a low energy: a negative pressure trace
    return u


@pytest.mark.parametrize("kind,p0,p1", [("toward_mean", 0.0, 0.0), ("toward_mean", 0.35, 0.0),
                                        ("toward_mean", 1.0, 0.0), ("positivity", 0.05, 0.05),
                                        ("positivity", 1e-13, 1e-13)])
def test_host_restatement_equals_the_oracle_traces(kind, p0, p1):
    orc = O.OracleSolver.one_d(p=3, nel=24, flux="hllc", method="persson", left="periodic", right="periodic")
    u = _spoiled_wave(orc)
    orc.set_state(u)
    orc.set_trace_override(kind, p0, p1)
    orc.residual()
    tl_ref, tr_ref = orc.traces_1d()
    ops = orc.ops()
    m = (F.TraceOverridePersson("toward_mean", theta=p0) if kind == "toward_mean"
         else F.TraceOverridePersson("positivity", eps_rho=p0, eps_p=p1))
    for e in range(orc.nel):
        tl, tr = m.element_traces(u[:, e, :], ops["w"], ops["l_L"], ops["l_R"], 1.4)
        assert np.allclose(tl, tl_ref[e], rtol=1e-14, atol=1e-14)
        assert np.allclose(tr, tr_ref[e], rtol=1e-14, atol=1e-14)


def test_positivity_traces_are_admissible_and_leave_good_elements_alone():
    orc = O.OracleSolver.one_d(p=3, nel=24, flux="hllc", method="persson", left="periodic", right="periodic")
    u = _spoiled_wave(orc)
    orc.set_state(u)
    orc.residual()
    plain = orc.traces_1d()
    orc.set_trace_override("positivity", 0.05, 0.05)
    orc.residual()
    lim = orc.traces_1d()

    def pres(t):
        return 0.4 * (t[:, 2] - 0.5 * t[:, 1] ** 2 / t[:, 0])

    for t in lim:
        assert (t[:, 0] >= 0.05 - 1e-14).all() and (pres(t) >= 0.05 - 1e-12).all()
    good = [e for e in range(orc.nel) if all(t[e, 0] >= 0.05 and pres(t[e:e + 1])[0] >= 0.05 for t in plain)]
    assert len(good) > 15
    for a, b in zip(plain, lim):
        assert np.array_equal(a[good], b[good])
    assert not np.array_equal(plain[0], lim[0])
