"""Pin the host restatement of the reference's 1D scoring metrics
(oracle/oracle_metrics.py: shock_thickness_sp, overshoot_metric,
smooth_region_mask + excess_dissipation, L1 against the exact Sod density
or the frozen Shu-Osher reference) against the scoring fields that the
reference recorded for its Sod and Shu-Osher cases
(test/data/snapshot_fixture/{baseline,method}.json, extracted by
tests/golden/make_golden.py), plus small known answers of
shock_thickness_sp's branches.

The recorded states are reproduced by the C oracle (n_steps and extrema,
test_oracle_golden.py); the fixture predates the current reference code, so
the floating-point fields agree at rounding level of the states, and the
thickness, a ratio of sample positions, exactly up to the last bits."""
import math
import os

import numpy as np
import pytest

import oracle as O
import oracle_metrics as M

O.set_threads(os.cpu_count() or 1)

SOD_WINDOWS = [(0.45, 0.55), (0.65, 0.95)]


def _samples(s):
    x = s.coords().ravel(order="F")
    rho = s.u[:, :, 0].ravel(order="F")
    return x, rho


@pytest.mark.parametrize("which,c_av", [("baseline", 0.1), ("method", 0.5)])
def test_sod_scoring_fields(golden, which, c_av):
    c = next(v for k, v in golden["snapshot_fixture"][which]["cases"].items() if k.startswith("sod"))
    s = O.OracleSolver.one_d(p=2, nel=64, method="persson", c_av=c_av)
    s.ic_sod()
    assert s.integrate(0.2, cfl=0.15)["n_steps"] == c["n_steps"]
    x, rho = _samples(s)
    assert np.all(np.diff(x) > 0)  # sample_solution_1d's sort is the identity
    assert M.shock_thickness_sp(x, rho) == pytest.approx(c["shock_thickness"], rel=1e-12)
    _, _, eta = M.overshoot_metric(rho.min(), rho.max(), 0.125, 1.0)
    assert eta == pytest.approx(c["overshoot"], abs=1e-9)
    rho_ex = M.sod_exact_density(x, 0.2)
    mask = M.smooth_region_mask(x, rho_ex, grad_frac=0.15, exclude_windows=SOD_WINDOWS)
    assert M.excess_dissipation(rho, rho_ex, mask) == pytest.approx(c["excess_dissipation_vs_exact"], rel=1e-7)
    assert M.l1_relative(rho, rho_ex) == pytest.approx(c["l1_density_vs_exact"], rel=1e-8)
    # the same case with NullCapturing
    n = O.OracleSolver.one_d(p=2, nel=64, method="null")
    n.ic_sod()
    assert n.integrate(0.2, cfl=0.15)["status"] == "ok"
    _, rho_n = _samples(n)
    mask_n = M.smooth_region_mask(x, rho_n, grad_frac=0.15, exclude_windows=SOD_WINDOWS)
    assert M.excess_dissipation(rho, rho_n, mask_n) == pytest.approx(c["excess_dissipation_vs_null"], rel=1e-6)
    assert c["excess_dissipation"] == c["excess_dissipation_vs_null"]


@pytest.mark.parametrize("which,c_av", [("baseline", 0.3), ("method", 0.5)])
def test_shu_osher_scoring_fields(golden, which, c_av):
    c = next(v for k, v in golden["snapshot_fixture"][which]["cases"].items() if k.startswith("shu_osher"))
    s = O.OracleSolver.one_d(p=1, nel=100, xl=0.0, xr=10.0, method="persson", c_av=c_av)
    s.ic_shu_osher()
    lo0, hi0 = s.extrema(0)
    assert s.integrate(1.8, cfl=0.1)["n_steps"] == c["n_steps"]
    x, rho = _samples(s)
    assert M.shock_thickness_sp(x, rho) == pytest.approx(c["shock_thickness"], rel=1e-12)
    _, _, eta = M.overshoot_metric(rho.min(), rho.max(), lo0, max(hi0, 4.5))
    assert eta == c["overshoot"] == 0.0
    ref = np.array(golden["shu_osher_ref"]["x_rho"])
    rho_ref = M.interp_1d(ref[:, 0], ref[:, 1], x)
    assert M.l1_relative(rho, rho_ref) == pytest.approx(c["l1_error_vs_reference"], rel=1e-7)
    n = O.OracleSolver.one_d(p=1, nel=100, xl=0.0, xr=10.0, method="null")
    n.ic_shu_osher()
    assert n.integrate(1.8, cfl=0.1)["status"] == "ok"
    xn, rho_n = _samples(n)
    mask = M.smooth_region_mask(x, rho_n, grad_frac=0.12, exclude_windows=[(1.5, 3.0)])
    # on the same mesh interp_1d returns the samples themselves
    assert np.array_equal(M.interp_1d(xn, rho_n, x), rho_n)
    assert M.excess_dissipation(rho, rho_n, mask) == pytest.approx(c["excess_dissipation"], rel=1e-6)


def test_shock_thickness_known_answers():
    # a rising profile whose values avoid the 10 % / 90 % levels: the walk
    # stops at 0.05 and 0.95, four spacings apart
    ramp = np.array([0.0] * 10 + [0.05, 0.3, 0.5, 0.7, 0.95] + [1.0] * 10)
    xr = np.arange(ramp.size, dtype=np.float64)
    assert M.steepest_gradient(xr, ramp)[0] == 11
    assert M.shock_thickness_sp(xr, ramp) == 4.0
    # the falling profile has the same thickness
    assert M.shock_thickness_sp(xr, 1.0 - ramp) == 4.0
    # a single-cell jump
    x = np.linspace(0.0, 1.0, 101)
    step = np.where(x < 0.5, 1.0, 0.125)
    assert M.shock_thickness_sp(x, step) == pytest.approx(1.0, rel=1e-12)
    # no jump, and fewer than four samples
    assert math.isnan(M.shock_thickness_sp(x, np.ones_like(x)))
    assert math.isnan(M.shock_thickness_sp(x[:3], step[:3]))
    # first index wins among equal gradients
    two = np.where(x < 0.3, 0.0, 1.0) + np.where(x < 0.7, 0.0, 1.0)
    assert M.steepest_gradient(x, two)[0] == int(np.argmax(x >= 0.3))


def test_overshoot_and_mask_semantics():
    assert M.overshoot_metric(0.1, 1.1, 0.125, 1.0) == pytest.approx((0.1 / 0.875, 0.025 / 0.875, 0.1 / 0.875))
    assert M.overshoot_metric(0.2, 0.9, 0.125, 1.0) == (0.0, 0.0, 0.0)
    assert all(math.isnan(v) for v in M.overshoot_metric(float("nan"), 1.0, 0.125, 1.0)[1:])
    x = np.linspace(0.0, 1.0, 11)
    rho = np.where(x < 0.5, 1.0, 0.5)
    m = M.smooth_region_mask(x, rho, grad_frac=0.1, exclude_windows=[(0.0, 0.1)])
    assert list(m) == [False, False, True, True, True, False, True, True, True, True, True]
