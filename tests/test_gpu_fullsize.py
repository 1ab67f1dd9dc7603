"""Parity at the benchmark sizes.

* The 512^2 P=3 HLLC + Persson BR0 workload (the bench's case): two SSP-RK3
  steps on the GPU against the oracle on the same seeded state.
* The 128^2 P=4 Rusanov + Persson periodic density wave: 100 steps against
  the oracle, and conservation of every component's discrete mass (periodic
  domain) measured on the GPU state with the device diagnostics.

The oracle runs with all host threads; each case takes seconds on the host.
"""
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


def test_128sq_p4_periodic_100_steps_and_mass():
    st, m = C2.build(F)
    orc = _oracle_for(C2)
    orc.set_state(st.u)
    mass0 = [orc.discrete_mass(c) for c in range(4)]
    r_ref = orc.integrate(1e9, cfl=C2.cfl, max_steps=100)
    s = F.GpuSolve(st, F.Euler2D(1.4), m)
    s.upload(st.u, 0.0)
    r = s.advance(1e9, cfl=C2.cfl, max_steps=100)
    assert r["status"] == r_ref["status"] and r["n_steps"] == r_ref["n_steps"] == 100
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
