"""The extrapolate_interface hook slot on the GPU.

A src/methods-style plugin (TraceOverridePersson) replaces the Lagrange
traces that the 1D interface fluxes use (extrapolate_interface!, called in
residual!, src/fr/Residual.jl:175; default Interfaces.jl:49-71) with a
device implementation ("traces_toward_mean", "traces_positivity_zhang_shu").
The oracle applies the same override where the reference calls the hook, so:

* the 1D residual with the override matches the oracle to 1e-12 on
  identical inputs (the reference's tables through the ABI), for both
  implementations, several parameters, boundary conditions, fluxes and
  dissipation forms;
* theta = 1 agrees with the default traces to rounding, and the positivity
  traces on an admissible state change nothing;
* an integration with the override matches the oracle (relative L1 1e-8,
  identical step counts) and differs from the run without it;
* the 2D residual ignores the slot, as the reference's never calls the hook;
* a batched 1D instance with the override matches the single solve.
"""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200.batch import Batch

from pairs import pair_1d, pair_2d, four_quadrant_state, rel_linf

pytestmark = pytest.mark.gpu


def _method(kind, p0, p1=1e-13, av_form="conservative_br0"):
    if kind == "toward_mean":
        return F.TraceOverridePersson("toward_mean", theta=p0, av_form=av_form)
    return F.TraceOverridePersson("positivity", eps_rho=p0, eps_p=p1, av_form=av_form)


def _spoiled_wave(orc):
    orc.ic_density_wave()
    u = orc.u.copy()
    u[0, 3, 0] = 0.02
    u[3, 8, 0] = 0.01
    u[1, 14, 2] *= 0.05
    return u


@pytest.mark.parametrize("kind,p0,p1", [("toward_mean", 0.0, 0.0), ("toward_mean", 0.35, 0.0),
                                        ("positivity", 0.05, 0.05)])
@pytest.mark.parametrize("bc", ["periodic", "transmissive", ("dirichlet", (1.0, 0.2, 2.6))])
@pytest.mark.parametrize("flux,av_form", [("hllc", "conservative_br0"), ("rusanov", "element_local_DD")])
def test_residual_with_trace_override_matches_oracle(kind, p0, p1, bc, flux, av_form):
    orc, state, _ = pair_1d(p=3, nel=24, flux=flux, method="persson", av_form=av_form, caller_ops=True,
                            left=bc, right=bc)
    u = _spoiled_wave(orc)
    orc.set_state(u)
    orc.t = 0.0
    orc.set_trace_override(kind, p0, p1)
    ref = orc.residual()
    s = F.GpuSolve(state, F.Euler1D(1.4), _method(kind, p0, p1, av_form), caller_ops=orc.ops())
    s.upload(u, 0.0)
    got = s.residual()
    assert rel_linf(got, ref) <= 1e-12
    orc.set_trace_override(None)
    assert rel_linf(orc.residual(), ref) > 1e-6  # the override changes the residual
    s.close()


def test_unit_theta_and_admissible_positivity_equal_the_default_traces():
    orc, state, plain = pair_1d(p=4, nel=40, flux="hllc", method="persson", left="periodic", right="periodic")
    orc.ic_density_wave()
    u = orc.u.copy()
    plain.upload(u, 0.0)
    r0 = plain.residual()
    for m in (_method("toward_mean", 1.0), _method("positivity", 1e-13, 1e-13)):
        s = F.GpuSolve(state, F.Euler1D(1.4), m)
        s.upload(u, 0.0)
        assert rel_linf(s.residual(), r0) <= 1e-15
        s.close()


# theta well below 1 is not a stable scheme with the FR correction: the
# oracle's Sod run diverges at theta = 0.5 (step 2394) and 0 (step 17)
@pytest.mark.parametrize("kind,p0", [("toward_mean", 0.9), ("positivity", 1e-3)])
def test_integration_with_trace_override_matches_oracle(kind, p0):
    orc, state, _ = pair_1d(p=3, nel=64, flux="hllc", method="persson")
    orc.ic_sod()
    u = orc.u.copy()
    orc.set_trace_override(kind, p0, p0)
    r_ref = orc.integrate(0.1, cfl=0.1)
    s = F.GpuSolve(state, F.Euler1D(1.4), _method(kind, p0, p0))
    s.upload(u, 0.0)
    r = s.advance(0.1, cfl=0.1)
    got, t = s.download()
    assert r["status"] == r_ref["status"] == "ok" and r["n_steps"] == r_ref["n_steps"]
    assert t == pytest.approx(orc.t, rel=1e-12)
    assert float(np.sum(np.abs(got - orc.u)) / np.sum(np.abs(orc.u))) <= 1e-8
    if kind == "toward_mean":
        orc2, state2, plain = pair_1d(p=3, nel=64, flux="hllc", method="persson")
        plain.upload(u, 0.0)
        plain.advance(0.1, cfl=0.1)
        assert rel_linf(plain.download()[0], got) > 1e-6  # the plugin changed the run
    s.close()


def test_2d_residual_ignores_the_slot():
    orc, state, plain = pair_2d(p=3, nx=10, ny=8, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc, jump_scale=0.25)
    plain.upload(u, 0.0)
    r0 = plain.residual()
    s = F.GpuSolve(state, F.Euler2D(1.4), _method("toward_mean", 0.2))
    s.upload(u, 0.0)
    assert np.array_equal(s.residual(), r0)
    s.close()


def test_batched_instance_with_trace_override():
    orc, state, _ = pair_1d(p=2, nel=48, flux="hllc", method="persson")
    orc.ic_sod()
    u = orc.u.copy()
    m = _method("toward_mean", 0.9)
    s = F.GpuSolve(state, F.Euler1D(1.4), m)
    s.upload(u, 0.0)
    r_ref = s.advance(0.05, cfl=0.1)
    ref, _ = s.download()
    b = Batch(capacity=2)
    i = b.add(state, F.Euler1D(1.4), m)
    b.upload(i, u, 0.0)
    b.start(i, 0.05, cfl=0.1)
    res = b.run()
    assert res[i]["status"] == r_ref["status"] and res[i]["n_steps"] == r_ref["n_steps"]
    assert rel_linf(b.download(i)[0], ref) <= 1e-10
    assert b.hook_calls(i)["extrapolate_interface"] is None
    b.close()
    s.close()
