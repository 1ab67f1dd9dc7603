"""The numerical_flux_method hook slot on the GPU.

A src/methods-style plugin (FluxOverridePersson) overrides the 1D interface
flux with a device implementation ("flux_rusanov" with a dissipation scale,
"flux_hllc").  The oracle resolves the same override where the reference
does (_resolve_flux, src/fr/Residual.jl:9-15), so:

* the 1D residual with the override matches the oracle to 1e-12 on
  identical inputs (the reference's tables through the ABI), for a Rusanov
  override under an HLLC scheme and the reverse;
* a Rusanov override with alpha = 1 is bit-identical to the scheme's own
  Rusanov flux;
* a shocked 1D integration with the override matches the oracle (relative
  L1 1e-8, identical step counts) and differs from the run without it;
* the 2D residual ignores the override, as the reference's does;
* a batched 1D instance with the override matches the single solve.
"""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200.batch import Batch

from pairs import pair_1d, pair_2d, four_quadrant_state, rel_linf

pytestmark = pytest.mark.gpu


def _plugin_solve(state, flux, alpha, eq=None):
    m = F.FluxOverridePersson(flux=flux, alpha=alpha)
    return F.GpuSolve(state, eq or F.Euler1D(1.4), m), m


@pytest.mark.parametrize("scheme_flux,override,alpha", [("hllc", "rusanov", 0.6), ("hllc", "rusanov", 1.7),
                                                        ("rusanov", "hllc", 1.0)])
@pytest.mark.parametrize("bc", ["transmissive", "periodic"])
def test_residual_with_flux_override_matches_oracle(scheme_flux, override, alpha, bc):
    orc, state, _ = pair_1d(p=3, nel=24, flux=scheme_flux, method="persson", caller_ops=True, left=bc, right=bc)
    orc.ic_sod() if bc == "transmissive" else orc.ic_density_wave()
    u = orc.u.copy()
    orc.set_flux_override(override, alpha)
    ref = orc.residual()
    m = F.FluxOverridePersson(flux=override, alpha=alpha)
    s = F.GpuSolve(state, F.Euler1D(1.4), m, caller_ops=orc.ops())
    s.upload(u, 0.0)
    got = s.residual()
    assert rel_linf(got, ref) <= 1e-12
    orc.set_flux_override(None)
    assert rel_linf(orc.residual(), ref) > 1e-6  # the override changes the residual
    s.close()


def test_unit_scale_equals_the_schemes_rusanov_bitwise():
    orc, state, plain = pair_1d(p=2, nel=30, flux="rusanov", method="persson")
    orc.ic_sod()
    u = orc.u.copy()
    plain.upload(u, 0.0)
    r0 = plain.residual()
    orc2, state2, _ = pair_1d(p=2, nel=30, flux="hllc", method="persson")
    s, _ = _plugin_solve(state2, "rusanov", 1.0)
    s.upload(u, 0.0)
    assert np.array_equal(s.residual(), r0)
    s.close()


def test_integration_with_flux_override_matches_oracle():
    orc, state, _ = pair_1d(p=3, nel=64, flux="hllc", method="persson")
    orc.ic_sod()
    u = orc.u.copy()
    orc.set_flux_override("rusanov", 0.8)
    r_ref = orc.integrate(0.1, cfl=0.1)
    s, _ = _plugin_solve(state, "rusanov", 0.8)
    s.upload(u, 0.0)
    r = s.advance(0.1, cfl=0.1)
    got, t = s.download()
    assert r["status"] == r_ref["status"] == "ok" and r["n_steps"] == r_ref["n_steps"]
    assert t == pytest.approx(orc.t, rel=1e-12)
    assert float(np.sum(np.abs(got - orc.u)) / np.sum(np.abs(orc.u))) <= 1e-8
    orc2, state2, plain = pair_1d(p=3, nel=64, flux="hllc", method="persson")
    plain.upload(u, 0.0)
    plain.advance(0.1, cfl=0.1)
    assert rel_linf(plain.download()[0], got) > 1e-6  # the plugin changed the run
    s.close()


def test_2d_residual_ignores_the_override():
    orc, state, plain = pair_2d(p=3, nx=10, ny=8, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc, jump_scale=0.25)
    plain.upload(u, 0.0)
    r0 = plain.residual()
    s, _ = _plugin_solve(state, "rusanov", 0.5, eq=F.Euler2D(1.4))
    s.upload(u, 0.0)
    assert np.array_equal(s.residual(), r0)
    s.close()


def test_batched_instance_with_flux_override():
    orc, state, _ = pair_1d(p=2, nel=48, flux="hllc", method="persson")
    orc.ic_sod()
    u = orc.u.copy()
    s, m = _plugin_solve(state, "rusanov", 0.7)
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
    b.close()
    s.close()
