"""Device-side set-up: case initial conditions evaluated on the device
(frg_set_initial_condition) against the oracle's restatement of the
reference ICs on the same mesh -- piecewise-constant states exactly, smooth
ones to the few-ulp differences of the device's sin/exp/pow -- and served
requests admitted with a device IC, bit-identical to the same request run
alone in a batch.  The analytic wavy metrics, also built on the device, are
covered by the curved residual parity tests of test_gpu_parity.py."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200.batch import Batch
from frforge_b200.serve import Server
from frforge_b200.workloads import four_quadrant_states, served_trace

from pairs import pair_1d, pair_2d, rel_linf

pytestmark = pytest.mark.gpu

SMOOTH_TOL = 1e-14


def _device(solve, **ic):
    solve.set_initial_condition(**ic)
    u, t = solve.download()
    assert t == 0.0
    return u


def test_sod_two_state_exact():
    orc, state, solve = pair_1d(p=3, nel=50)
    orc.ic_sod()
    u = _device(solve, kind="two_state", prim=[(1.0, 0.0, 1.0), (0.125, 0.0, 0.1)], x0=0.5)
    assert np.array_equal(u, orc.u)


def test_shu_osher_and_density_wave_1d():
    orc, state, solve = pair_1d(p=4, nel=64, xl=0.0, xr=10.0)
    orc.ic_shu_osher()
    u = _device(solve, kind="shu_osher")
    assert rel_linf(u, orc.u) <= SMOOTH_TOL
    orc, state, solve = pair_1d(p=2, nel=40, left="periodic", right="periodic")
    orc.ic_density_wave(0.03)
    u = _device(solve, kind="density_wave", prim=[(1.0, 1.0, 1.0)], amp=0.2, t=0.03)
    assert rel_linf(u, orc.u) <= SMOOTH_TOL


def test_four_quadrant_exact():
    orc, state, solve = pair_2d(p=3, nx=11, ny=9, bcs=("transmissive",) * 4)
    ne, nw, sw, se = four_quadrant_states(77, 0.25)
    orc.ic_four_quadrant(ne, nw, sw, se, 0.5, 0.5)
    u = _device(solve, kind="four_quadrant", prim=[ne, nw, sw, se], x0=0.5, y0=0.5)
    assert np.array_equal(u, orc.u)


def test_vortex_and_smooth_2d():
    orc, state, solve = pair_2d(p=4, nx=10, ny=10, xl=0.0, xr=10.0, yb=0.0, yt=10.0)
    orc.ic_vortex(0.25)
    u = _device(solve, kind="vortex", t=0.25)
    assert rel_linf(u, orc.u) <= SMOOTH_TOL
    orc, state, solve = pair_2d(p=3, nx=8, ny=8, wavy=1, amp=0.05)
    orc.ic_smooth_2d()
    u = _device(solve, kind="smooth_2d")
    assert rel_linf(u, orc.u) <= SMOOTH_TOL


def test_invalid_ic():
    orc, state, solve = pair_1d(p=2, nel=8)
    with pytest.raises(ValueError):
        solve.set_initial_condition(kind="vortex")
    orc, state, solve = pair_2d(p=2, nx=4, ny=4)
    with pytest.raises(ValueError):
        solve.set_initial_condition(kind="shu_osher")


def test_served_with_device_ic_matches_solo():
    trace = served_trace(seed=13, count=8, n2d=(6, 20), n1d=(24, 160), t_final=(0.005, 0.02))
    srv = Server(slots=4, steps_per_pump=8)
    ids = []
    for req in trace:
        st, eq, m = req.build(F)
        ids.append(srv.submit_ic(st, eq, req.ic(), m, t_final=req.t_final, cfl=req.cfl))
    srv.drain()
    for rid, req in zip(ids, trace):
        res = srv.result(rid)
        assert res["status"] == "ok"
        st, eq, m = req.build(F)
        b = Batch(capacity=1)
        i = b.add(st, eq, m)
        b.set_initial_condition(i, **req.ic())
        b.start(i, req.t_final, cfl=req.cfl)
        r = b.run()[i]
        u, t = b.download(i)
        b.close()
        assert res["n_steps"] == r["n_steps"] and res["t"] == r["t"]
        assert np.array_equal(res["u"], u)
        # the device IC is the host-built one up to the device's sin
        st2, _, _ = req.build(F)
        s = F.GpuSolve(st2, eq, m)
        s.set_initial_condition(**req.ic())
        u_dev, _ = s.download()
        assert rel_linf(u_dev, st2.u) <= SMOOTH_TOL
    srv.close()
