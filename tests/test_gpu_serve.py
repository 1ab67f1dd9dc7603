"""Served execution (frg_server_*): a seeded request trace, admitted into a
batch as slots free up.  Every delivered result is bit-identical to the same
request run alone in a batch (its result does not depend on what else is
being served, on arrival order, on admission waits or on multirate
scheduling), and agrees with the single-solve path to 1e-10."""
import dataclasses

import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200 import _lib as L
from frforge_b200.batch import Batch, solve_bytes
from frforge_b200.serve import Server
from frforge_b200.workloads import served_trace

from pairs import rel_linf

pytestmark = pytest.mark.gpu


def small_trace(count=12, seed=7):
    return served_trace(seed=seed, count=count, n2d=(6, 20), n1d=(24, 160), t_final=(0.005, 0.02))


def solo(req):
    st, eq, m = req.build(F)
    b = Batch(capacity=1)
    i = b.add(st, eq, m)
    b.start(i, req.t_final, cfl=req.cfl)
    r = b.run()[i]
    u, t = b.download(i)
    b.close()
    return r, u


def single(req):
    st, eq, m = req.build(F)
    s = F.GpuSolve(st, eq, m)
    s.upload(st.u, 0.0)
    r = s.advance(req.t_final, cfl=req.cfl)
    u, _ = s.download()
    s.close()
    return r, u


def check(res, req):
    r_solo, u_solo = solo(req)
    assert res["status"] == r_solo["status"] and res["n_steps"] == r_solo["n_steps"]
    assert res["t"] == r_solo["t"]
    assert np.array_equal(res["u"], u_solo)
    r_one, u_one = single(req)
    assert res["n_steps"] == r_one["n_steps"] and res["status"] == r_one["status"]
    assert rel_linf(res["u"], u_one) <= 1e-10


def test_trace_all_at_once():
    trace = small_trace()
    srv = Server(slots=5, steps_per_pump=8)
    ids = [srv.submit(*req.build(F), t_final=req.t_final, cfl=req.cfl) for req in trace]
    srv.drain()
    done = srv.take_completed()
    assert sorted(done) == sorted(ids)
    for rid, req in zip(ids, trace):
        res = srv.result(rid)
        assert res["status"] == "ok"
        check(res, req)
    srv.close()


def test_trace_in_waves_with_cancel():
    trace = small_trace(count=10, seed=11)
    srv = Server(slots=3, steps_per_pump=4)
    ids = []
    for k, req in enumerate(trace):
        ids.append(srv.submit(*req.build(F), t_final=req.t_final, cfl=req.cfl))
        if k % 3 == 2:
            srv.pump()
    # cancel one that may be running (or done already), and one still queued
    srv.cancel(ids[4])
    srv.cancel(ids[-1])
    srv.drain()
    for k, (rid, req) in enumerate(zip(ids, trace)):
        res = srv.result(rid)
        if k == len(ids) - 1 or (k == 4 and res["status"] == "cancelled"):
            assert res["status"] == "cancelled"
            continue
        check(res, req)
    srv.close()


def test_budget_limits_concurrency():
    # six requests of one size; the budget holds two of them at a time
    base = small_trace(count=1, seed=23)[0]
    trace = [dataclasses.replace(base, seed=base.seed + k) for k in range(6)]
    st, eq, m = base.build(F)
    one = F.GpuSolve(st, eq, m).info()["device_bytes"]
    sizes = [solve_bytes(*req.build(F)) for req in trace]
    assert min(sizes) >= one
    srv = Server(slots=6, hbm_budget=int(2.5 * one), steps_per_pump=4)
    ids = [srv.submit(*req.build(F), t_final=req.t_final, cfl=req.cfl) for req in trace]
    peak = 0
    while True:
        _, q, a = srv.pump()
        peak = max(peak, a)
        if q == 0 and a == 0:
            break
    assert peak <= 2
    for rid, req in zip(ids, trace):
        check(srv.result(rid), req)
    srv.close()
    # a request larger than the whole budget is refused at submit
    srv = Server(slots=2, hbm_budget=one // 4)
    with pytest.raises(F.FRGError) as e:
        srv.submit(*base.build(F), t_final=base.t_final)
    assert e.value.code == L.FRG_ERR_OOM
    srv.close()


def test_divergent_request_isolated():
    trace = small_trace(count=4, seed=31)
    srv = Server(slots=4, steps_per_pump=8)
    ids = []
    for k, req in enumerate(trace):
        st, eq, m = req.build(F)
        if k == 2:
            st.u.flat[5] = np.nan
        ids.append(srv.submit(st, eq, m, t_final=req.t_final, cfl=req.cfl))
    srv.drain()
    for k, (rid, req) in enumerate(zip(ids, trace)):
        res = srv.result(rid)
        if k == 2:
            assert res["status"] == "diverged"
        else:
            check(res, req)
    srv.close()


def test_multirate_batch_matches_lockstep():
    trace = small_trace(count=8, seed=41)
    b = Batch(capacity=8)
    b.set_multirate(True)
    slots = []
    for req in trace:
        st, eq, m = req.build(F)
        i = b.add(st, eq, m)
        b.start(i, req.t_final, cfl=req.cfl)
        slots.append(i)
    res = b.run()
    for i, req in zip(slots, trace):
        r_solo, u_solo = solo(req)
        assert res[i] == r_solo
        u, _ = b.download(i)
        assert np.array_equal(u, u_solo)
    b.close()


def test_diagnostics_without_state_download():
    # want_state=False: the final state stays on the device; the delivered
    # diagnostics equal those of the same request run alone in a batch
    trace = small_trace(count=5, seed=61)
    srv = Server(slots=3, steps_per_pump=8)
    ids = [srv.submit(*req.build(F), t_final=req.t_final, cfl=req.cfl, want_state=False) for req in trace]
    srv.drain()
    for rid, req in zip(ids, trace):
        res = srv.result(rid)
        assert res["u"] is None and res["status"] == "ok"
        st, eq, m = req.build(F)
        b = Batch(capacity=1)
        i = b.add(st, eq, m)
        b.start(i, req.t_final, cfl=req.cfl)
        b.run()
        ref = b.diagnostics(i)
        b.close()
        got = res["diagnostics"]
        assert got["mass"] == ref["mass"] and got["rho_min"] == ref["rho_min"]
        assert got["rho_max"] == ref["rho_max"] and got["p_min"] == ref["p_min"]
        assert got["positivity_ok"] and got["nonfinite"] == 0 and got["t"] == ref["t"]
    srv.close()
