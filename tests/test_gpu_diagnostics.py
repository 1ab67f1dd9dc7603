"""Device-side diagnostics (frg_diagnostics_compute) against the oracle's
restatement of the reference's scoring reductions on the same state:
discrete_mass, density extrema, positivity_ok, has_nonfinite and l2_error
with the vortex, smooth 2D and 1D density-wave exact solutions.  Sums are
reduced in a different order on the device, so they agree to 1e-12
relative; extrema, counts and flags agree exactly."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200.batch import Batch

from pairs import four_quadrant_state, pair_1d, pair_2d, prim2cons1, prim2cons2, smooth_state_2d

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _check_common(d, orc, neq):
    for c in range(neq):
        ref = orc.discrete_mass(c)
        assert abs(d["mass"][c] - ref) <= TOL * max(abs(ref), 1e-300), (c, d["mass"][c], ref)
    lo, hi = orc.extrema(0)
    assert d["rho_min"] == lo and d["rho_max"] == hi
    assert d["positivity_ok"] == orc.positivity_ok()
    assert (d["nonfinite"] > 0) == orc.has_nonfinite()


def test_vortex_2d_mass_extrema_l2():
    orc, state, solve = pair_2d(p=3, nx=12, ny=12, xl=0.0, xr=10.0, yb=0.0, yt=10.0)
    orc.ic_vortex(0.0)
    solve.upload(orc.u.copy(), 0.0)
    for t_exact in (0.0, 0.4):
        d = solve.diagnostics(exact="vortex_2d", t_exact=t_exact)
        _check_common(d, orc, 4)
        ref = orc.l2_error_vortex(t_exact)
        assert abs(d["l2_error"] - ref) <= TOL * max(ref, 1e-14) + 1e-15, (d["l2_error"], ref)
        assert d["nonfinite"] == 0 and d["positivity_ok"]


def test_smooth_2d_on_wavy_mesh():
    orc, state, solve = pair_2d(p=4, nx=8, ny=8, wavy=1, amp=0.05)
    orc.ic_smooth_2d()
    u = orc.u.copy()
    solve.upload(u, 0.0)
    d = solve.diagnostics(exact="smooth_2d", t_exact=0.1)
    _check_common(d, orc, 4)
    ref = orc.l2_error_smooth_2d(0.1)
    assert abs(d["l2_error"] - ref) <= TOL * ref


def test_density_wave_1d_l2_and_mass():
    orc, state, solve = pair_1d(p=3, nel=40, left="periodic", right="periodic")
    orc.ic_density_wave(0.0)
    solve.upload(orc.u.copy(), 0.0)
    d = solve.diagnostics(exact="density_wave_1d", t_exact=0.05, c=0)
    _check_common(d, orc, 3)
    ref = orc.l2_error_density_wave(0.05)
    assert abs(d["l2_error"] - ref) <= TOL * ref


def test_positivity_and_nonfinite_flags():
    orc, state, solve = pair_2d(p=2, nx=6, ny=5, bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc, jump_scale=0.25)
    u[1, 2, 7, 0] = -0.5  # negative density at one point
    orc.set_state(u)
    solve.upload(u, 0.0)
    d = solve.diagnostics()
    _check_common(d, orc, 4)
    assert not d["positivity_ok"] and d["rho_min"] == -0.5
    u[0, 0, 3, 3] = np.nan
    u[2, 1, 9, 1] = np.inf
    orc.set_state(u)
    solve.upload(u, 0.0)
    d = solve.diagnostics()
    assert d["nonfinite"] == 2 and not d["positivity_ok"]
    assert np.isnan(d["mass"][3]) and not np.isnan(d["mass"][0])


def test_reference_state_l2_and_batched_instance():
    torch = pytest.importorskip("torch")
    orc, state, solve = pair_2d(p=3, nx=10, ny=10, method="persson")
    u0 = smooth_state_2d(orc, seed=5)
    state.u[...] = u0
    # advance 10 steps in a batch, then compare its state with the initial one
    b = Batch(capacity=1)
    i = b.add(state, F.Euler2D(1.4), F.PerssonAVMethod())
    b.start(i, 1.0, cfl=0.1, max_steps=10)
    b.run()
    u, t = b.download(i)
    d = b.diagnostics(i)
    orc.set_state(u)
    _check_common(d, orc, 4)
    assert d["t"] == t
    # L2 difference against a reference state in device memory (component 2)
    ref = torch.tensor(np.asarray(u0).ravel(order="F"), dtype=torch.float64, device="cuda")
    solve.upload(u, t)
    d2 = solve.diagnostics(exact="state", ref_ptr=ref.data_ptr(), c=2)
    w = np.asarray(orc.ops()["w"])
    J = np.abs(orc.metric("J"))
    ww = w[:, None, None] * w[None, :, None] * J
    expect = np.sqrt(np.sum(ww * (u[..., 2] - u0[..., 2]) ** 2))
    assert abs(d2["l2_error"] - expect) <= TOL * expect
    b.close()


def test_invalid_requests():
    orc, state, solve = pair_1d(p=2, nel=8)
    orc.ic_sod()
    solve.upload(orc.u.copy(), 0.0)
    with pytest.raises(ValueError):
        solve.diagnostics(exact="vortex_2d")  # 2D exact solution on a 1D solve
    with pytest.raises(ValueError):
        solve.diagnostics(c=3)  # 1D has 3 components
    with pytest.raises(ValueError):
        solve.diagnostics(exact="state")  # no reference pointer
