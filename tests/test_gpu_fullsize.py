"""Parity at the benchmark sizes and lengths.

* The 512^2 P=3 HLLC + Persson BR0 workload (the bench's case, seeded
  four-quadrant IC with jump_scale 0.25):
  - two SSP-RK3 steps against the oracle on the same state (tight bar);
  - 100 steps against the oracle: relative L1 <= 1e-8 with identical status,
    step count, positivity and non-finite flags (the shocked-case bar);
  - its full 1000 steps against the oracle's recorded summary of the same
    run (tests/golden/c3_oracle_summary.json, written by
    tests/golden/make_c3_summary.py): step counts, times, discrete masses,
    density extrema and flags at steps 100, 250, 500 and 1000, from the
    device diagnostics.
* The 128^2 P=4 Rusanov + Persson periodic density wave for its full 500
  steps against the oracle (smooth-case bar 1e-9), and conservation of every
  component's discrete mass measured on the GPU state.

The oracle runs with all host threads; the longest case (100 steps of the
512^2 workload) takes about half a minute on 16 host threads.
"""
import json
import math
import os

import numpy as np
import pytest

import frforge_b200 as F
import oracle as O
from frforge_b200.workloads import C1, C2, C3

pytestmark = pytest.mark.gpu


def _oracle_for(w):
    bc = "periodic" if w.periodic else "transmissive"
    O.set_threads(os.cpu_count() or 1)
    return O.OracleSolver.two_d(p=w.p, nx=w.n, ny=w.n, bcs=[O.make_bc(bc)] * 4, flux=w.flux, method="persson",
                                c_av=w.c_av)


def _rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


def test_512sq_p3_hllc_two_steps():
    st, m = C3.build(F)
    orc = _oracle_for(C3)
    orc.set_state(st.u)
    r_ref = orc.integrate(1e9, cfl=C3.cfl, max_steps=2)
    s = F.GpuSolve(st, F.Euler2D(1.4), m)
    s.upload(st.u, 0.0)
    r = s.advance(1e9, cfl=C3.cfl, max_steps=2)
    u, t = s.download()
    assert r["status"] == r_ref["status"] == "max_steps" and r["n_steps"] == 2
    assert t == pytest.approx(orc.t, rel=1e-13)
    assert _rel_l1(u, orc.u) <= 1e-12
    assert np.max(np.abs(u - orc.u)) / np.max(np.abs(orc.u)) <= 1e-10


def test_512sq_p3_hllc_100_steps():
    st, m = C3.build(F)
    orc = _oracle_for(C3)
    orc.set_state(st.u)
    r_ref = orc.integrate(1e9, cfl=C3.cfl, max_steps=100)
    s = F.GpuSolve(st, F.Euler2D(1.4), m)
    s.upload(st.u, 0.0)
    r = s.advance(1e9, cfl=C3.cfl, max_steps=100)
    d = s.diagnostics()
    u, t = s.download()
    assert r["status"] == r_ref["status"] == "max_steps" and r["n_steps"] == r_ref["n_steps"] == 100
    assert t == pytest.approx(orc.t, rel=1e-12)
    assert _rel_l1(u, orc.u) <= 1e-8
    assert d["positivity_ok"] == orc.positivity_ok()
    assert (d["nonfinite"] > 0) == orc.has_nonfinite() == False  # noqa: E712


def _c3_summary():
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c3_oracle_summary.json")) as f:
        return json.load(f)


def test_512sq_p3_hllc_1000_steps_against_oracle_summary():
    ref = _c3_summary()
    st, m = C3.build(F)
    s = F.GpuSolve(st, F.Euler2D(1.4), m)
    s.upload(st.u, 0.0)
    # shocked flow: rounding differences grow over the run (the masses agree
    # to ~1e-10 at step 500 and ~5e-9 at step 1000), so the integrals take
    # the shocked-case bar 1e-8 and the pointwise extrema 1e-7; step counts,
    # status and flags are exact
    done, bad = 0, []
    for cp in ref["checkpoints"]:
        r = s.advance(1e9, cfl=C3.cfl, max_steps=cp["n_steps"] - done)
        done += r["n_steps"]
        d = s.diagnostics()
        assert r["status"] == cp["status"] and done == cp["n_steps"], (r, cp)
        assert d["positivity_ok"] == cp["positivity_ok"]
        assert (d["nonfinite"] > 0) == cp["nonfinite"]
        checks = [("t", d["t"], cp["t"], 1e-12)]
        checks += [(f"mass[{c}]", d["mass"][c], cp["mass"][c], 1e-8) for c in range(4)]
        checks += [("rho_min", d["rho_min"], cp["rho_min"], 1e-7), ("rho_max", d["rho_max"], cp["rho_max"], 1e-7)]
        for name, got, want, tol in checks:
            err = abs(got - want) / max(abs(want), 1e-300)
            if err > tol:
                bad.append((done, name, got, want, err))
    assert not bad, bad
    assert done == 1000


def test_128sq_p4_periodic_500_steps_and_mass():
    st, m = C2.build(F)
    orc = _oracle_for(C2)
    orc.set_state(st.u)
    mass0 = [orc.discrete_mass(c) for c in range(4)]
    r_ref = orc.integrate(1e9, cfl=C2.cfl, max_steps=C2.steps)
    s = F.GpuSolve(st, F.Euler2D(1.4), m)
    s.upload(st.u, 0.0)
    r = s.advance(1e9, cfl=C2.cfl, max_steps=C2.steps)
    assert r["status"] == r_ref["status"] and r["n_steps"] == r_ref["n_steps"] == C2.steps == 500
    d = s.diagnostics()
    u, t = s.download()
    assert t == pytest.approx(orc.t, rel=1e-12)
    assert np.max(np.abs(u - orc.u)) / np.max(np.abs(orc.u)) <= 1e-9
    # periodic domain: the FR scheme conserves every component
    for c in range(4):
        assert abs(d["mass"][c] - mass0[c]) <= 1e-12 * max(abs(mass0[c]), 1.0), c
    assert d["positivity_ok"] and d["nonfinite"] == 0


def test_c1_1d_full_length():
    # the 1D case at its full length: 256 elements, P=3, 2000 SSP-RK3 steps
    st, m = C1.build(F)
    O.set_threads(os.cpu_count() or 1)
    orc = O.OracleSolver.one_d(p=C1.p, nel=C1.nel, flux=C1.flux, method="persson", c_av=C1.c_av)
    orc.set_state(st.u)
    r_ref = orc.integrate(1e9, cfl=C1.cfl, max_steps=C1.steps)
    s = F.GpuSolve(st, F.Euler1D(1.4), m)
    s.upload(st.u, 0.0)
    r = s.advance(1e9, cfl=C1.cfl, max_steps=C1.steps)
    u, t = s.download()
    assert r["status"] == r_ref["status"] == "max_steps" and r["n_steps"] == r_ref["n_steps"] == C1.steps
    assert t == pytest.approx(orc.t, rel=1e-12)
    # shocked state: relative L1 to 1e-8
    assert _rel_l1(u, orc.u) <= 1e-8


def test_c2_smooth_order_p4():
    # run_euler2d_smooth_order (src/verification/Cases2D_Smooth.jl:94-150) at
    # P=4: NullCapturing, t_final 0.25, fixed dt from the finest mesh
    # (dt = cfl/(p+1) h/((2p+1) lambda), lambda = 1 + sqrt(gamma), cfl 0.06),
    # the smooth wave evaluated and measured on the device; observed orders
    # must reach formal - 0.3 (order_pass, src/verification/Metrics.jl:34-45).
    # At P=4 the density L2 error meets the FP64 round-off floor of the time
    # loop (about 1.3e-12 after 21,000 steps, measured at n = 128 and 256), so
    # the meshes are n = 16..64, whose errors lie above it (n = 8 is still
    # pre-asymptotic: order 4.69 from 8 to 16).  Measured orders 4.91, 4.97.
    p, n_list, t_final, cfl, gamma = 4, [16, 32, 64], 0.25, 0.06, 1.4
    lam = 1.0 + math.sqrt(gamma)
    dt = (cfl / (p + 1)) * (1.0 / max(n_list)) / ((2 * p + 1) * lam)
    errs = []
    for n in n_list:
        bc = F.PeriodicBC
        mesh = F.Mesh2D(0.0, 1.0, 0.0, 1.0, n, n, bc(), bc(), bc(), bc())
        st = F.allocate_state(mesh, F.build_operators(p), 4)
        s = F.GpuSolve(st, F.Euler2D(gamma), F.NullCapturing())
        s.set_initial_condition("smooth_2d")
        r = s.advance(t_final, dt=dt)
        assert r["status"] == "ok", n
        d = s.diagnostics(exact="smooth_2d", t_exact=t_final)
        assert d["t"] == pytest.approx(t_final, abs=1e-14) and d["nonfinite"] == 0
        errs.append(d["l2_error"])
        s.close()
    assert errs[-1] > 1e-11  # above the round-off floor
    orders = [math.log(errs[k] / errs[k + 1]) / math.log(2.0) for k in range(len(errs) - 1)]
    assert all(q >= (p + 1) - 0.3 for q in orders), (errs, orders)
