"""GPU parity: the CUDA path through the C ABI against the C oracle.

Tolerances are the stated bar: residual relative L-infinity <= 1e-12
(absolute when the reference residual is ~0, as for freestream), smooth
final states <= 1e-9, shocked final states <= 1e-8 in relative L1 with
identical status / positivity flags and step counts.
"""
import math

import numpy as np
import pytest

import frforge_b200 as F
from pairs import (four_quadrant_state, pair_1d, pair_2d, prim2cons1, prim2cons2, rel_linf,
                   smooth_state_2d, splitmix64)

pytestmark = pytest.mark.gpu

RES_TOL = 1e-12


def _residual_pair(orc, state, solve, u, t=0.0):
    orc.set_state(u)
    orc.t = t
    ref = orc.residual()
    solve.upload(u, t)
    got = solve.residual()
    return got, ref


CASES_2D = [
    dict(p=1, method="null"),
    dict(p=2, method="null", flux="hllc"),
    dict(p=3, method="persson", flux="hllc", bcs=("transmissive",) * 4),
    dict(p=4, method="persson"),
    dict(p=5, method="persson", flux="hllc"),
    dict(p=3, method="persson", av_form="element_local_DD"),
    dict(p=3, points="gll", method="persson", flux="hllc"),
    dict(p=2, method="persson", bcs=("reflecting", "transmissive", "reflecting", "transmissive")),
    dict(p=2, method="null", flux="hllc",
         bcs=(("dirichlet", (1.0, 0.5, 0.1, 2.6)), "transmissive", "periodic", "periodic")),
    dict(p=3, nx=9, ny=7, method="persson", flux="hllc", bcs=("transmissive",) * 4),
    dict(p=2, nx=5, ny=3, method="persson", bcs=("periodic",) * 4),
]


@pytest.mark.parametrize("cfg", CASES_2D, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items() if k != "bcs"))
@pytest.mark.parametrize("ic", ["smooth", "shock"])
def test_residual_2d(cfg, ic):
    # identical inputs: the reference's operator tables and its (D-differentiated)
    # metric arrays go through the ABI
    orc, state, solve = pair_2d(caller_ops=True, gpu_metrics=True, **cfg)
    u = smooth_state_2d(orc) if ic == "smooth" else four_quadrant_state(orc)
    got, ref = _residual_pair(orc, state, solve, u)
    assert np.all(np.isfinite(got))
    assert rel_linf(got, ref) <= RES_TOL, rel_linf(got, ref)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("ic", ["smooth", "shock"])
def test_residual_2d_affine_path(p, ic):
    # the production path: library-built tables (Newton GL nodes, ~1 ulp from
    # the reference's eigen-based nodes) and exact affine metrics (the
    # reference differentiates x(xi) with D, which leaves ~1e-14 relative
    # error in x_xi, y_eta at P=5); agreement is then a few 1e-12 of max|du|
    orc, state, solve = pair_2d(p=p, method="persson", flux="hllc", bcs=("transmissive",) * 4)
    u = smooth_state_2d(orc) if ic == "smooth" else four_quadrant_state(orc)
    got, ref = _residual_pair(orc, state, solve, u)
    assert rel_linf(got, ref) <= 1e-11


def test_residual_2d_caller_tables_and_metrics():
    # reference tables and D-differentiated metrics handed over unchanged
    orc, state, solve = pair_2d(p=3, method="persson", flux="hllc", gpu_metrics=True, caller_ops=True,
                                bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc)
    got, ref = _residual_pair(orc, state, solve, u)
    assert rel_linf(got, ref) <= RES_TOL


@pytest.mark.parametrize("geom", ["wavy-analytic", "wavy-metrics"])
def test_residual_2d_curved(geom):
    orc, state, solve = pair_2d(p=3, nx=6, ny=5, method="persson", wavy=1, amp=0.05,
                                gpu_metrics=(geom == "wavy-metrics"), caller_ops=True)
    u = smooth_state_2d(orc)
    got, ref = _residual_pair(orc, state, solve, u)
    assert rel_linf(got, ref) <= RES_TOL


def test_residual_2d_solid_mask():
    # forward-facing-step style solid block with reflecting walls
    nx, ny = 12, 6
    solid = np.zeros(nx * ny, dtype=bool)
    for jy in range(2):
        for jx in range(4, nx):
            solid[jy * nx + jx] = True
    orc, state, solve = pair_2d(p=2, nx=nx, ny=ny, method="persson", flux="hllc", solid=solid,
                                caller_ops=True, gpu_metrics=True,
                                bcs=(("dirichlet", (1.4, 4.2, 0.0, 2.5 + 0.5 * 1.4 * 9)), "transmissive",
                                     "reflecting", "reflecting"))
    u = smooth_state_2d(orc)
    got, ref = _residual_pair(orc, state, solve, u)
    assert rel_linf(got, ref) <= RES_TOL
    blk = got.reshape(-1, nx * ny, 4, order="F")
    assert np.all(blk[:, solid, :] == 0.0)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_tile_variants_agree(p):
    # every tile variant of the stage kernel is a separate instantiation
    orc, state, solve = pair_2d(p=p, nx=11, ny=9, method="persson", flux="hllc", caller_ops=True,
                                gpu_metrics=True, bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc)
    orc.set_state(u)
    ref = orc.residual()
    _, n = solve.variant()
    assert n >= 2
    for v in range(n):
        solve.set_variant(v)
        solve.upload(u, 0.0)
        assert rel_linf(solve.residual(), ref) <= RES_TOL, v
    solve.upload(u, 0.0)
    best, ms = solve.autotune(reps=2)
    assert 0 <= best < n and np.all(ms > 0)
    assert solve.variant()[0] == best


def test_freestream_residual_2d():
    # test/test_2d.jl:304-315 (residual max < 1e-12)
    orc, state, solve = pair_2d(p=2, nx=4, ny=4)
    x, _ = orc.coords()
    u = prim2cons2(np.ones_like(x), 0.5 + 0 * x, 0.25 + 0 * x, 1.0 + 0 * x)
    solve.upload(u, 0.0)
    assert np.max(np.abs(solve.residual())) < 1e-12


CASES_1D = [
    dict(p=1, method="null"),
    dict(p=2, method="persson", flux="hllc"),
    dict(p=3, method="persson"),
    dict(p=4, method="persson", av_form="element_local_DD"),
    dict(p=5, method="persson", flux="hllc", left="periodic", right="periodic"),
    dict(p=3, points="gll", method="persson", left=("dirichlet", (1.0, 0.2, 2.6)),
         right=("dirichlet", (0.125, 0.0, 0.25))),
    dict(p=2, nel=100, method="persson", flux="hllc"),
]


@pytest.mark.parametrize("cfg", CASES_1D, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
def test_residual_1d(cfg):
    orc, state, solve = pair_1d(caller_ops=True, **cfg)
    x = orc.coords()
    g = splitmix64(11)
    ph = [2 * np.pi * next(g) for _ in range(3)]
    r = np.where(x < 0.5, 1.0, 0.125) + 0.05 * np.sin(2 * np.pi * x + ph[0])
    u = prim2cons1(r, 0.2 * np.sin(2 * np.pi * x + ph[1]), np.where(x < 0.5, 1.0, 0.1) + 0 * x)
    got, ref = _residual_pair(orc, state, solve, u)
    assert rel_linf(got, ref) <= RES_TOL, rel_linf(got, ref)


def test_sensor_2d_and_dt():
    orc, state, solve = pair_2d(p=3, method="persson", flux="hllc", bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc)
    orc.set_state(u)
    solve.upload(u, 0.0)
    s_ref = orc.sense()
    s_got = solve.sense()
    assert np.max(np.abs(s_got - s_ref)) <= 1e-12 * max(1.0, np.max(s_ref))
    assert solve.compute_dt(0.1) == pytest.approx(orc.compute_dt(0.1), rel=1e-14)


def test_residual_deterministic():
    # test/test_threading.jl:14-47: two residual calls give identical du
    orc, state, solve = pair_2d(p=3, method="persson", flux="hllc", bcs=("transmissive",) * 4)
    u = four_quadrant_state(orc)
    solve.upload(u, 0.0)
    a = solve.residual()
    b = solve.residual()
    assert np.array_equal(a, b)


def test_sod_integration_matches_oracle(golden):
    # Sod p=2 Ne=64 persson_av, snapshot fixture: 950 steps
    c = golden["snapshot_fixture"]["baseline"]["cases"]["sod_p2_ne64_persson_av"]
    orc, state, solve = pair_1d(p=2, nel=64, method="persson", c_av=0.1)
    orc.ic_sod()
    u0 = orc.u.copy()
    r_ref = orc.integrate(0.2, cfl=0.15)
    solve.upload(u0, 0.0)
    r = solve.advance(0.2, cfl=0.15)
    u, t = solve.download()
    assert r["status"] == "ok" and r["n_steps"] == r_ref["n_steps"] == c["n_steps"]
    assert t == pytest.approx(0.2, abs=1e-15)
    ref = orc.u
    assert np.sum(np.abs(u - ref)) / np.sum(np.abs(ref)) <= 1e-8
    assert abs(u[:, :, 0].min() - c["u_min"]) < 1e-8 and abs(u[:, :, 0].max() - c["u_max"]) < 1e-8


def test_vortex_golden_gpu(golden):
    # isentropic vortex L2 (test/test_2d.jl:316-321) through the GPU path
    v = golden["vortex"]
    p, L = v["p"], 10.0
    lam = 1.0 + 1.0 + 5.0 / (2 * math.pi) + math.sqrt(1.4) + 1.0
    dt = (v["cfl"] / (p + 1)) * (L / max(v["n_list"])) / ((2 * p + 1) * lam)
    errs = []
    for n in v["n_list"]:
        orc, state, solve = pair_2d(p=p, nx=n, ny=n, xl=0.0, xr=L, yb=0.0, yt=L)
        orc.ic_vortex(0.0)
        solve.upload(orc.u.copy(), 0.0)
        r = solve.advance(v["t_final"], dt=dt)
        assert r["status"] == "ok"
        u, _ = solve.download()
        orc.set_state(u)
        errs.append(orc.l2_error_vortex(v["t_final"]))
    for got, ref in zip(errs, v["l2_errors"]):
        assert abs(got - ref) <= 1e-9 * abs(ref)
    order = math.log(errs[0] / errs[1]) / math.log(2.0)
    assert abs(order - v["observed_order"]) <= 1e-8


def test_shocked_2d_integration_matches_oracle():
    # small four-quadrant HLLC + Persson BR0 case (the 512^2 benchmark's physics)
    orc, state, solve = pair_2d(p=3, nx=24, ny=24, flux="hllc", method="persson",
                                bcs=("transmissive",) * 4)
    u0 = four_quadrant_state(orc, jump_scale=0.25)
    orc.set_state(u0)
    r_ref = orc.integrate(1.0, cfl=0.1, max_steps=60)
    solve.upload(u0, 0.0)
    r = solve.advance(1.0, cfl=0.1, max_steps=60)
    u, t = solve.download()
    assert r["status"] == r_ref["status"] == "max_steps"
    assert r["n_steps"] == r_ref["n_steps"] == 60
    assert t == pytest.approx(orc.t, rel=1e-12)
    ref = orc.u
    assert np.sum(np.abs(u - ref)) / np.sum(np.abs(ref)) <= 1e-8
    orc.set_state(u)
    assert orc.positivity_ok()


def test_unscaled_draw_diverges_at_same_step():
    # the unscaled seeded four-quadrant draw drives the reference scheme to
    # negative density; the GPU must report :diverged at the same step with
    # the same state
    orc, state, solve = pair_2d(p=3, nx=16, ny=16, flux="hllc", method="persson",
                                bcs=("transmissive",) * 4)
    u0 = four_quadrant_state(orc)
    orc.set_state(u0)
    r_ref = orc.integrate(10.0, cfl=0.1, max_steps=200)
    solve.upload(u0, 0.0)
    r = solve.advance(10.0, cfl=0.1, max_steps=200)
    assert r_ref["status"] == r["status"] == "diverged"
    assert r["n_steps"] == r_ref["n_steps"]
    u, t = solve.download()
    assert t == pytest.approx(orc.t, rel=1e-12)


def test_smooth_2d_rk2_fixed_dt():
    orc, state, solve = pair_2d(p=4, nx=8, ny=8, method="persson", time="ssp_rk2")
    u0 = smooth_state_2d(orc)
    orc.set_state(u0)
    r_ref = orc.integrate(0.05, dt=1e-3)
    solve.upload(u0, 0.0)
    r = solve.advance(0.05, dt=1e-3)
    u, _ = solve.download()
    assert r["n_steps"] == r_ref["n_steps"] and r["status"] == "ok"
    assert rel_linf(u, orc.u) <= 1e-9


def test_divergence_flag_matches_oracle():
    orc, state, solve = pair_1d(p=2, nel=16, method="null")
    x = orc.coords()
    u = prim2cons1(1.0 + 0 * x, 0 * x, 1.0 + 0 * x)
    u[1, 5, 0] = np.nan
    orc.set_state(u)
    r_ref = orc.integrate(0.1, cfl=0.1)
    solve.upload(u, 0.0)
    r = solve.advance(0.1, cfl=0.1)
    assert r["status"] == r_ref["status"] == "diverged"
    assert r["n_steps"] == r_ref["n_steps"]


def test_python_api_roundtrip():
    # the reference-shaped API: allocate_state / set_initial_condition_ / integrate_
    eq = F.Euler1D(1.4)
    ops = F.build_operators(2)
    mesh = F.Mesh1D(0.0, 1.0, 64, F.TransmissiveBC(), F.TransmissiveBC())
    st = F.allocate_state(mesh, ops, 3)
    F.set_initial_condition_(st, lambda x: eq.primitives_to_conserved(
        np.where(x < 0.5, 1.0, 0.125), 0.0 * x, np.where(x < 0.5, 1.0, 0.1)))
    r = F.integrate_(st, eq, F.get_capturing_method("persson_av"), 0.2, cfl=0.15)
    assert r["status"] == "ok" and r["n_steps"] == 950
    assert F.positivity_ok(eq, st)
    du = np.zeros_like(st.u)
    F.residual_(du, st, eq, F.PerssonAVMethod())
    assert np.all(np.isfinite(du))


def test_unsupported_hook_raises():
    class CustomSense(F.PerssonAVMethod):
        def sense_(self, sigma, u_work, state, eq):
            return sigma

    eq = F.Euler1D(1.4)
    st = F.allocate_state(F.Mesh1D(0.0, 1.0, 8), F.build_operators(2), 3)
    with pytest.raises(F.UnsupportedHookError):
        F.integrate_(st, eq, CustomSense(), 0.01)


def test_hook_pipeline_counts():
    # test/test_capturing.jl:5-61: stages per step, via the device counters
    orc, state, solve = pair_1d(p=2, nel=8, method="persson", left="periodic", right="periodic")
    x = orc.coords()
    u = prim2cons1(1.0 + 0.1 * np.sin(2 * np.pi * x), 0.1 + 0 * x, 1.0 + 0 * x)
    solve.upload(u, 0.0)
    r = solve.advance(0.05, cfl=0.2)
    info = solve.info()
    assert info["steps"] == r["n_steps"] >= 1
    assert info["residual_evals"] == 3 * r["n_steps"]
