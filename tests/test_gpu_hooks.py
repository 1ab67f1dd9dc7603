"""Device hook registry: the Zhang-Shu post-step kernel against its host
restatement on identical states (1D, 2D affine, 2D wavy), and its place in
the device time loop against a host-driven loop of single steps with the
host hook in between.  Batched and served instances run the hook after each
of their completed steps: bit-identical to the instance alone in a batch and
within 1e-10 of the single-solve path (bit-identical for solo groups)."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200 import _lib as L
from frforge_b200.batch import Batch
from frforge_b200.gpu import set_solve_hooks
from frforge_b200.limiters import zhang_shu_limit_
from frforge_b200.serve import Server

from pairs import four_quadrant_state, pair_1d, pair_2d, rel_linf

pytestmark = pytest.mark.gpu


def _spoil_2d(u):
    u = u.copy()
    u[1, 2, 5, 0] = -0.04     # negative density
    u[0, 1, 9, 3] = 1e-3      # negative pressure
    u[2, 2, 14, 3] = 0.02
    return u


@pytest.mark.parametrize("wavy", [0, 1])
def test_kernel_matches_host_2d(wavy):
    orc, state, solve = pair_2d(p=3, nx=6, ny=5, flux="hllc", method="persson", wavy=wavy,
                                bcs=("transmissive",) * 4)
    u = _spoil_2d(four_quadrant_state(orc, jump_scale=0.25))
    m = F.PositivityPreservingPersson()
    s = F.GpuSolve(state, F.Euler2D(1.4), m)
    s.upload(u, 0.0)
    s.apply_post_step()
    got, _ = s.download()
    state.u[...] = u
    if wavy:
        state.metrics = {"J": orc.metric("J")}  # the host limiter's |J| at the points
    zhang_shu_limit_(state, F.Euler2D(1.4))
    assert rel_linf(got, state.u) <= 1e-13
    assert not np.array_equal(got, u)  # the spoiled elements were limited
    assert np.all(got[..., 0] > 0)


def test_kernel_matches_host_1d():
    orc, state, solve = pair_1d(p=4, nel=12)
    orc.ic_sod()
    u = orc.u.copy()
    u[2, 3, 0] = -0.01
    u[1, 8, 2] = 1e-4
    m = F.PositivityPreservingPersson()
    s = F.GpuSolve(state, F.Euler1D(1.4), m)
    s.upload(u, 0.0)
    s.apply_post_step()
    got, _ = s.download()
    state.u[...] = u
    zhang_shu_limit_(state, F.Euler1D(1.4))
    assert rel_linf(got, state.u) <= 1e-13


def test_time_loop_matches_host_driven_steps():
    # thresholds just below the initial minima: the hook clips the
    # undershoots at the shocks every step, away from vacuum
    orc, state, _ = pair_2d(p=3, nx=16, ny=16, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    u0 = four_quadrant_state(orc, jump_scale=0.25)
    eq = F.Euler2D(1.4)
    er = 0.98 * float(np.min(u0[..., 0]))
    ep = 0.98 * float(np.min(eq.pressure(u0)))
    nsteps, cfl = 12, 0.1
    m = F.PositivityPreservingPersson(eps_rho=er, eps_p=ep)
    dev = F.GpuSolve(state, eq, m)
    dev.upload(u0, 0.0)
    r = dev.advance(1e9, cfl=cfl, max_steps=nsteps)
    u_dev, t_dev = dev.download()
    # host-driven: one GPU step without the hook, then the host hook
    plain = F.GpuSolve(state, eq, F.PerssonAVMethod())
    u = u0.copy()
    t = 0.0
    for _ in range(nsteps):
        plain.upload(u, t)
        dt = plain.compute_dt(cfl)
        assert plain.step(dt) == "ok"
        u, t = plain.download()
        state.u[...] = u
        zhang_shu_limit_(state, eq, er, ep)
        u = state.u.copy()
    assert r["status"] == "max_steps" and r["n_steps"] == nsteps
    assert t_dev == pytest.approx(t, rel=1e-12)
    assert rel_linf(u_dev, u) <= 1e-10
    # the hook changed the run
    plain.upload(u0, 0.0)
    plain.advance(1e9, cfl=cfl, max_steps=nsteps)
    u_plain, _ = plain.download()
    assert rel_linf(u_plain, u_dev) > 1e-8
    assert np.min(u_dev[..., 0]) >= er * (1 - 1e-12) and np.min(u_plain[..., 0]) < er


def _hooked_cases():
    """(state, eq, hooked method, plain method, run) of the batch tests: the
    thresholds sit just below each initial state's minima, so the hook clips
    the undershoots at the discontinuities every step."""
    eq2, eq1 = F.Euler2D(1.4), F.Euler1D(1.4)
    out = []
    for k, (kw, scale) in enumerate([
            (dict(p=3, nx=16, ny=16, flux="hllc"), 0.25),
            (dict(p=2, nx=12, ny=10, flux="rusanov", time="ssp_rk2"), 0.25),
            (dict(p=2, nx=10, ny=10, flux="hllc", wavy=1), 0.2)]):
        orc, state, _ = pair_2d(method="persson", bcs=("transmissive",) * 4, **kw)
        u0 = four_quadrant_state(orc, seed=60 + k, jump_scale=scale)
        state.u[...] = u0
        state.t = 0.0
        er = 0.98 * float(np.min(u0[..., 0]))
        ep = 0.98 * float(np.min(eq2.pressure(u0)))
        out.append((state, eq2, F.PositivityPreservingPersson(eps_rho=er, eps_p=ep), F.PerssonAVMethod(),
                    dict(t_final=1.0, cfl=0.1, max_steps=10)))
    orc, state, _ = pair_1d(p=3, nel=48, method="persson")
    orc.ic_sod()
    state.u[...] = orc.u
    state.t = 0.0
    out.append((state, eq1, F.PositivityPreservingPersson(eps_rho=0.124, eps_p=0.099), F.PerssonAVMethod(),
                dict(t_final=1.0, cfl=0.15, max_steps=40)))
    return out


def _single(state, eq, m, run):
    s = F.GpuSolve(state, eq, m)
    s.upload(state.u, 0.0)
    r = s.advance(run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    u, t = s.download()
    s.close()
    return r, u, t


def _alone(state, eq, m, run):
    b = Batch(capacity=1)
    i = b.add(state, eq, m)
    b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    r = b.run()[i]
    u, t = b.download(i)
    b.close()
    return r, u, t


def test_batch_runs_post_step_hook_like_a_single_solve():
    # hooked instances (2D affine RK3/RK2, 2D wavy, 1D) beside their unhooked
    # twins in one batch: each ends bit-identical to itself alone in a batch,
    # within 1e-10 of the single-solve path with the hook, and away from the
    # unhooked run
    cases = _hooked_cases()
    b = Batch(capacity=2 * len(cases))
    slots = []
    for state, eq, mh, mp, run in cases:
        for m in (mh, mp):
            i = b.add(state, eq, m)
            b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
            slots.append(i)
    res = b.run()
    for k, (state, eq, mh, mp, run) in enumerate(cases):
        ih, ip = slots[2 * k], slots[2 * k + 1]
        uh, th = b.download(ih)
        up, _ = b.download(ip)
        r_alone, u_alone, t_alone = _alone(state, eq, mh, run)
        assert res[ih] == r_alone and th == t_alone and np.array_equal(uh, u_alone), k
        r_one, u_one, t_one = _single(state, eq, mh, run)
        assert res[ih]["status"] == r_one["status"] == "max_steps", k
        assert res[ih]["n_steps"] == r_one["n_steps"], k
        assert th == pytest.approx(t_one, rel=1e-13), k
        assert rel_linf(uh, u_one) <= 1e-10, k
        # the hook acted: the plain run breaks a floor that the hooked run
        # keeps, and the two runs differ
        assert np.min(uh[..., 0]) >= mh.eps_rho * (1 - 1e-12), k
        assert np.min(eq.pressure(uh)) >= mh.eps_p * (1 - 1e-9), k
        assert np.min(up[..., 0]) < mh.eps_rho or np.min(eq.pressure(up)) < mh.eps_p, k
        assert rel_linf(uh, up) > 1e-8, k
    b.close()


def test_solo_group_runs_post_step_hook():
    # 200^2 P=3 fills a wave of batched tiles and runs solo inside the batch,
    # through the single-solve kernels and hook: bit-identical to frg_advance
    orc, state, _ = pair_2d(p=3, nx=200, ny=200, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    u0 = four_quadrant_state(orc, seed=71, jump_scale=0.25)
    state.u[...] = u0
    state.t = 0.0
    eq = F.Euler2D(1.4)
    m = F.PositivityPreservingPersson(eps_rho=0.98 * float(np.min(u0[..., 0])),
                                      eps_p=0.98 * float(np.min(eq.pressure(u0))))
    run = dict(t_final=1.0, cfl=0.1, max_steps=6)
    r_one, u_one, t_one = _single(state, eq, m, run)
    b = Batch(capacity=2)
    i = b.add(state, eq, m)
    b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    r = b.run()[i]
    u, t = b.download(i)
    b.close()
    assert r["status"] == r_one["status"] and r["n_steps"] == r_one["n_steps"] == 6
    assert t == t_one and np.array_equal(u, u_one)


def test_hook_selected_between_runs_regroups_the_instance():
    # a plain run, then the same slot restarted after a hook was selected on
    # its solve: the second run is the hooked one
    state, eq, mh, mp, run = _hooked_cases()[0]
    b = Batch(capacity=2)
    i = b.add(state, eq, mp)
    b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    b.run()
    b.upload(i, state.u, 0.0)
    set_solve_hooks(b._solve(i), b.ctx, mh)
    b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    r = b.run()[i]
    u, t = b.download(i)
    b.close()
    r_alone, u_alone, t_alone = _alone(state, eq, mh, run)
    assert r == r_alone and t == t_alone and np.array_equal(u, u_alone)


def test_server_runs_post_step_hook():
    cases = _hooked_cases()
    srv = Server(slots=3, steps_per_pump=4)
    ids = []
    for state, eq, mh, mp, run in cases:
        ids.append(srv.submit(state, eq, mh, t_final=run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"]))
    srv.drain()
    for rid, (state, eq, mh, mp, run) in zip(ids, cases):
        res = srv.result(rid)
        r_alone, u_alone, t_alone = _alone(state, eq, mh, run)
        assert res["status"] == r_alone["status"] and res["n_steps"] == r_alone["n_steps"]
        assert res["t"] == t_alone and np.array_equal(res["u"], u_alone)
    # a hook for an admitted request, or an unknown one, is refused
    state, eq, mh, mp, run = cases[0]
    rid = srv.submit(state, eq, mp, t_final=run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    lib = L.load()
    par, bad = np.array([1e-3, 1e-3]), np.array([-1e-3, 1e-3])
    assert lib.frg_server_set_hook(srv.handle, rid, 0, 7, L.dptr(par), 2) == L.FRG_ERR_UNSUPPORTED_HOOK
    assert lib.frg_server_set_hook(srv.handle, rid, 0, 1, L.dptr(bad), 2) == L.FRG_ERR_INVALID_ARG
    srv.pump()
    assert lib.frg_server_set_hook(srv.handle, rid, 0, 1, L.dptr(par), 2) == L.FRG_ERR_STATE
    srv.drain()
    srv.close()


def test_multirate_batch_with_hooks_matches_alone():
    # multirate scheduling gives the groups different step counts per round;
    # hooked and plain instances still end as they do alone in a batch
    cases = _hooked_cases()
    b = Batch(capacity=2 * len(cases))
    b.set_multirate(True)
    slots = []
    for state, eq, mh, mp, run in cases:
        for m in (mh, mp):
            i = b.add(state, eq, m)
            b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
            slots.append((i, state, eq, m, run))
    res = b.run()
    for i, state, eq, m, run in slots:
        r_alone, u_alone, t_alone = _alone(state, eq, m, run)
        u, t = b.download(i)
        assert res[i] == r_alone and t == t_alone and np.array_equal(u, u_alone), i
    b.close()


def test_served_device_ic_with_hook_matches_alone():
    # a hooked request admitted with its initial state evaluated on the device
    orc, state, _ = pair_2d(p=2, nx=16, ny=16, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    eq = F.Euler2D(1.4)
    ic = dict(kind="four_quadrant", prim=[(1.0, 0.0, 0.0, 1.0), (0.5, 0.6, 0.0, 0.4), (0.15, 0.6, 0.6, 0.05),
                                           (0.3, 0.0, 0.6, 0.2)], x0=0.5, y0=0.5)
    m = F.PositivityPreservingPersson(eps_rho=0.14, eps_p=0.045)
    run = dict(t_final=1.0, cfl=0.1, max_steps=15)
    srv = Server(slots=2, steps_per_pump=4)
    rid = srv.submit_ic(state, eq, ic, m, t_final=run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    srv.drain()
    res = srv.result(rid)
    srv.close()
    b = Batch(capacity=1)
    i = b.add(state, eq, m)
    b.set_initial_condition(i, **ic)
    b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
    r = b.run()[i]
    u, t = b.download(i)
    b.close()
    assert res["status"] == r["status"] == "max_steps" and res["n_steps"] == r["n_steps"] == 15
    assert res["t"] == t and np.array_equal(res["u"], u)
    assert np.min(u[..., 0]) >= 0.14 * (1 - 1e-12)
