"""Device-side 1D scoring metrics (frg_shock_metrics_1d) against the host
restatement of src/verification/Metrics.jl (oracle/oracle_metrics.py,
itself pinned to the reference's recorded Sod / Shu-Osher scoring fields in
test_shock_metrics_host.py), evaluated on the same downloaded GPU state:
indices and the shock thickness exactly, the reduced sums to 1e-12; and
the GPU runs' fields against the recorded ones."""
import math

import numpy as np
import pytest

import oracle_metrics as M

from pairs import pair_1d

pytestmark = pytest.mark.gpu

SOD_WINDOWS = [(0.45, 0.55), (0.65, 0.95)]


def _x(solve_state):
    return solve_state.mesh.physical_coords(solve_state.ops).ravel(order="F")


def _run(p, nel, method, c_av, ic, t_final, cfl, xl=0.0, xr=1.0):
    orc, state, solve = pair_1d(p=p, nel=nel, method=method, c_av=c_av, xl=xl, xr=xr)
    getattr(orc, ic)()
    solve.upload(orc.u.copy(), 0.0)
    r = solve.advance(t_final, cfl=cfl)
    u, _ = solve.download()
    return state, solve, r, u[:, :, 0].ravel(order="F")


def _check_against_host(d, x, rho, ref, grad_frac, windows, ref_min, ref_max):
    assert d["n_samples"] == x.size
    imax, _ = M.steepest_gradient(x, rho)
    assert d["shock_index"] == imax and d["shock_x"] == x[imax]
    th = M.shock_thickness_sp(x, rho)
    assert (math.isnan(th) and math.isnan(d["shock_thickness"])) or d["shock_thickness"] == th
    assert d["rho_min"] == rho.min() and d["rho_max"] == rho.max()
    assert (d["overshoot_over"], d["overshoot_under"], d["overshoot"]) == M.overshoot_metric(
        rho.min(), rho.max(), ref_min, ref_max)
    if ref is None:
        assert d["excess_dissipation"] is None and d["l1_rel"] is None
        return
    mask = M.smooth_region_mask(x, ref, grad_frac=grad_frac, exclude_windows=windows)
    assert d["excess_dissipation"] == pytest.approx(M.excess_dissipation(rho, ref, mask), rel=1e-12)
    assert d["l1_rel"] == pytest.approx(M.l1_relative(rho, ref), rel=1e-12)


def test_sod_metrics_on_device(golden):
    c = golden["snapshot_fixture"]["baseline"]["cases"]["sod_p2_ne64_persson_av"]
    st, s, r, rho = _run(2, 64, "persson", 0.1, "ic_sod", 0.2, 0.15)
    assert r["status"] == "ok" and r["n_steps"] == c["n_steps"]
    stn, sn, rn, rho_n = _run(2, 64, "null", 0.1, "ic_sod", 0.2, 0.15)
    assert rn["status"] == "ok"
    x = _x(st)
    # against the NullCapturing run held on the device
    d = s.shock_metrics(ref=sn, ref_min=0.125, ref_max=1.0, grad_frac=0.15, exclude=SOD_WINDOWS)
    _check_against_host(d, x, rho, rho_n, 0.15, SOD_WINDOWS, 0.125, 1.0)
    assert d["shock_thickness"] == pytest.approx(c["shock_thickness"], rel=1e-12)
    assert d["overshoot"] == pytest.approx(c["overshoot"], abs=1e-8)
    assert d["excess_dissipation"] == pytest.approx(c["excess_dissipation_vs_null"], rel=1e-5)
    # against the exact density from the host
    rho_ex = M.sod_exact_density(x, 0.2)
    e = s.shock_metrics(ref=rho_ex, grad_frac=0.15, exclude=SOD_WINDOWS)
    _check_against_host(e, x, rho, rho_ex, 0.15, SOD_WINDOWS, 0.125, 1.0)
    assert e["excess_dissipation"] == pytest.approx(c["excess_dissipation_vs_exact"], rel=1e-6)
    assert e["l1_rel"] == pytest.approx(c["l1_density_vs_exact"], rel=1e-7)
    # no reference
    _check_against_host(s.shock_metrics(), x, rho, None, 0.15, (), 0.125, 1.0)


def test_shu_osher_metrics_on_device(golden):
    c = golden["snapshot_fixture"]["baseline"]["cases"]["shu_osher_p1_ne100_persson_av"]
    st, s, r, rho = _run(1, 100, "persson", 0.3, "ic_shu_osher", 1.8, 0.1, xr=10.0)
    assert r["n_steps"] == c["n_steps"]
    x = _x(st)
    ref = np.array(golden["shu_osher_ref"]["x_rho"])
    rho_ref = M.interp_1d(ref[:, 0], ref[:, 1], x)
    d = s.shock_metrics(ref=rho_ref, ref_min=0.0, ref_max=4.5, grad_frac=0.12, exclude=[(1.5, 3.0)])
    _check_against_host(d, x, rho, rho_ref, 0.12, [(1.5, 3.0)], 0.0, 4.5)
    assert d["shock_thickness"] == pytest.approx(c["shock_thickness"], rel=1e-12)
    assert d["l1_rel"] == pytest.approx(c["l1_error_vs_reference"], rel=1e-6)


def test_shock_metrics_arguments():
    st, s, _, _ = _run(2, 16, "persson", 0.1, "ic_sod", 0.01, 0.15)
    with pytest.raises(ValueError):
        s.shock_metrics(ref=np.ones(5))
    with pytest.raises(ValueError):
        s.shock_metrics(exclude=[(0, 1)] * 5)
    # invalid arguments are ValueError (FRG_ERR_INVALID_ARG), as the
    # reference's ArgumentError
    with pytest.raises(ValueError, match="window_sp"):
        s.shock_metrics(window_sp=0)
    _, other, _, _ = _run(2, 20, "null", 0.1, "ic_sod", 0.01, 0.15)
    with pytest.raises(ValueError, match="other samples"):
        s.shock_metrics(ref=other)
    from pairs import pair_2d
    _, st2, s2 = pair_2d(p=2, nx=4, ny=4)
    s2.upload(np.ones(st2.u.shape), 0.0)
    with pytest.raises(ValueError, match="1D"):
        s2.shock_metrics()
