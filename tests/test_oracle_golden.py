"""Pin the CPU oracle against the reference's own recorded results.

Every number compared here comes from the reference's tests or fixtures
(extracted by tests/golden/make_golden.py): test/test_2d.jl:304-321,
test/data/snapshot_fixture/*.json and test/data/shu_osher_ref.csv.  The
operator checks restate test/test_operators.jl and test/test_schemes.jl.
"""
import math
import os

import numpy as np
import pytest

import oracle as O

O.set_threads(os.cpu_count() or 1)


@pytest.mark.parametrize("points", ["gl", "gll"])
@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_operators_known_answers(p, points):
    # test/test_operators.jl:5-60, test/test_schemes.jl:19-52
    ops = O.build_operators(p, points)
    xi, w, D = ops["xi"], ops["w"], ops["D"]
    assert np.all(np.diff(xi) > 0) and np.all(np.abs(xi) <= 1)
    assert abs(w.sum() - 2) < 1e-12
    assert abs((w * xi).sum()) < 1e-13
    tol = 1e-12 if points == "gl" else 1e-10
    for k in range(p + 1):
        ex = np.zeros_like(xi) if k == 0 else k * xi ** (k - 1)
        assert np.allclose(D @ xi**k, ex, atol=tol, rtol=tol)
    assert abs(ops["l_L"].sum() - 1) < 1e-13 and abs(ops["l_R"].sum() - 1) < 1e-13
    assert np.all(np.isfinite(ops["gL_xi"])) and np.all(np.isfinite(ops["gR_xi"]))
    if points == "gll":
        assert abs(xi[0] + 1) < 1e-15 and abs(xi[-1] - 1) < 1e-15
        assert abs(ops["l_L"][0] - 1) < 1e-12 and abs(ops["l_R"][-1] - 1) < 1e-12


def test_gdg_endpoints():
    # g_DG endpoints: g_L(-1)=1, g_L(1)=0, g_R(-1)=0, g_R(1)=1 (test_operators.jl:38-51)
    for p in range(1, 6):
        gll = O.build_operators(p, "gll")  # GLL nodes include the endpoints
        assert abs(gll["gL"][0] - 1) < 1e-12 and abs(gll["gL"][-1]) < 1e-12
        assert abs(gll["gR"][0]) < 1e-12 and abs(gll["gR"][-1] - 1) < 1e-12


def test_hllc_stationary_contact():
    # test/test_schemes.jl:88-103
    g = 1.4
    uL = [1.0, 0.0, 1.0 / (g - 1)]
    uR = [0.1, 0.0, 1.0 / (g - 1)]
    fh = O.flux_1d("hllc", g, uL, uR)
    assert abs(fh[1] - 1.0) < 1e-10
    assert np.all(np.isfinite(O.flux_1d("rusanov", g, [1, 0, 2.5], [0.125, 0, 0.25])))


def _vortex(n, g):
    v = g["vortex"]
    p, L = v["p"], 10.0
    lam = 1.0 + 1.0 + 5.0 / (2 * math.pi) + math.sqrt(1.4) + 1.0
    h = L / max(v["n_list"])
    dt = (v["cfl"] / (p + 1)) * h / ((2 * p + 1) * lam)
    s = O.OracleSolver.two_d(p=p, nx=n, ny=n, xl=0, xr=L, yb=0, yt=L)
    s.ic_vortex(0.0)
    r = s.integrate(v["t_final"], dt=dt)
    assert r["status"] == "ok"
    return s.l2_error_vortex(v["t_final"])


def test_vortex_l2_golden(golden):
    # test/test_2d.jl:316-321 (rtol 1e-12 / 1e-10)
    v = golden["vortex"]
    e = [_vortex(n, golden) for n in v["n_list"]]
    for got, ref in zip(e, v["l2_errors"]):
        assert abs(got - ref) <= v["rtol_l2"] * abs(ref) + 1e-14
    order = math.log(e[0] / e[1]) / math.log(2.0)
    assert abs(order - v["observed_order"]) <= v["rtol_order"] * abs(v["observed_order"]) + 1e-12


def test_freestream_cartesian_residual():
    # test/test_2d.jl:304-315: freestream residual < 1e-12
    s = O.OracleSolver.two_d(p=2, nx=4, ny=4)
    s.ic_uniform([1.0, 0.5, 0.25, 1.0])
    assert np.max(np.abs(s.residual())) < 1e-12


def test_freestream_curved_residual():
    # test/test_2d.jl:102-111: analytic wavy metrics, residual < 5e-4
    s = O.OracleSolver.two_d(p=3, nx=4, ny=4, wavy=1, amp=0.05)
    s.ic_uniform([1.0, 0.5, 0.25, 1.0])
    assert np.max(np.abs(s.residual())) < 5e-4
    assert np.all(s.metric("J") > 0)


@pytest.mark.parametrize("case", ["euler_smooth_order_p2", "euler_smooth_order_p3"])
def test_smooth_order_1d_golden(golden, case):
    c = golden["snapshot_fixture"]["baseline"]["cases"][case]
    p = c["p"]
    nlist = c["n_elements_list"]
    dt = (0.1 / (p + 1)) * (1.0 / max(nlist)) / ((2 * p + 1) * 2.5)
    assert dt == c["dt_fixed"]
    for ne, ref in zip(nlist, c["l2_errors"]):
        s = O.OracleSolver.one_d(p=p, nel=ne, left="periodic", right="periodic")
        s.ic_density_wave(0.0)
        assert s.integrate(1.0, dt=dt)["status"] == "ok"
        got = s.l2_error_density_wave(1.0)
        # the fixture predates the current code; agreement is at rounding level
        assert abs(got - ref) <= 1e-10 * abs(ref) + 1e-14


@pytest.mark.parametrize("which,c_av", [("baseline", 0.1), ("method", 0.5)])
def test_sod_golden(golden, which, c_av):
    cases = golden["snapshot_fixture"][which]["cases"]
    c = next(v for k, v in cases.items() if k.startswith("sod"))
    s = O.OracleSolver.one_d(p=2, nel=64, method="persson", c_av=c_av)
    s.ic_sod()
    m0 = s.discrete_mass(0)
    r = s.integrate(0.2, cfl=0.15)
    lo, hi = s.extrema(0)
    assert r["status"] == "ok" and r["n_steps"] == c["n_steps"]
    assert abs(lo - c["u_min"]) < 1e-10 and abs(hi - c["u_max"]) < 1e-10
    assert abs((s.discrete_mass(0) - m0) - c["mass_change"]) < 1e-11
    assert s.positivity_ok()


@pytest.mark.parametrize("which,c_av", [("baseline", 0.3), ("method", 0.5)])
def test_shu_osher_golden(golden, which, c_av):
    cases = golden["snapshot_fixture"][which]["cases"]
    c = next(v for k, v in cases.items() if k.startswith("shu_osher"))
    assert c["method_params"]["c_av"] == c_av
    s = O.OracleSolver.one_d(p=1, nel=100, xl=0.0, xr=10.0, method="persson", c_av=c_av)
    s.ic_shu_osher()
    r = s.integrate(1.8, cfl=0.1)
    lo, hi = s.extrema(0)
    assert r["n_steps"] == c["n_steps"]
    assert abs(lo - c["u_min"]) < 1e-10 and abs(hi - c["u_max"]) < 1e-10


def test_shu_osher_reference_csv(golden):
    g = golden["shu_osher_ref"]
    ref = np.array(g["x_rho"])
    s = O.OracleSolver.one_d(p=g["p"], nel=g["ne"], xl=0.0, xr=10.0, method="persson", c_av=g["c_av"])
    s.ic_shu_osher()
    assert s.integrate(g["t_final"], cfl=g["cfl"])["status"] == "ok"
    x = s.coords().ravel(order="F")
    rho = s.u[:, :, 0].ravel(order="F")
    assert np.array_equal(x, ref[:, 0])
    assert np.max(np.abs(rho - ref[:, 1])) < 1e-10
    assert np.sum(np.abs(rho - ref[:, 1])) / np.sum(np.abs(ref[:, 1])) < 1e-11


def test_br0_annihilates_constants():
    # test/test_capturing.jl:86-90 and test/test_2d.jl:47: BR0 on a constant state
    s1 = O.OracleSolver.one_d(p=3, nel=8, left="periodic", right="periodic", method="persson", c_av=1.0)
    s1.ic_uniform([1.0, 0.3, 1.0])
    du = s1.residual()
    ops = s1.ops()
    mass = sum(ops["w"][j] * (1.0 / 16) * du[j, e, 0] for e in range(8) for j in range(4))
    assert abs(mass) < 1e-12
    s2 = O.OracleSolver.two_d(p=2, nx=4, ny=4, method="persson", c_av=1.0)
    s2.ic_uniform([1.0, 0.3, -0.2, 1.0])
    assert np.max(np.abs(s2.residual())) < 1e-10


def test_serial_bit_determinism():
    # test/test_threading.jl:14-47 (two residual calls give identical du)
    s = O.OracleSolver.two_d(p=2, nx=4, ny=4, method="persson", c_av=0.1)
    x, y = s.coords()
    u = s.u
    u[..., 0] = 1.0 + 0.1 * np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y)
    u[..., 1] = 0.1 * u[..., 0]
    u[..., 2] = -0.05 * u[..., 0]
    u[..., 3] = 1.0 / 0.4 + 0.5 * u[..., 0] * (0.01 + 0.0025)
    assert np.array_equal(s.residual(), s.residual())


def test_sensor_activates_on_jump():
    # test/test_2d.jl:44-66
    s = O.OracleSolver.two_d(p=2, nx=4, ny=4, method="persson", c_av=0.1)
    x, y = s.coords()
    g = 1.4
    hi = np.array([1.0, 0.0, 0.0, 1.0 / (g - 1)])
    lo = np.array([0.125, 0.0, 0.0, 0.1 / (g - 1)])
    mask = (x + y) < 0.7
    for c in range(4):
        s.u[..., c] = np.where(mask, hi[c], lo[c])
    sig = s.sense()
    assert np.all((sig >= 0) & (sig <= 1)) and sig.max() > 0.01
    assert np.all(np.isfinite(s.residual()))
