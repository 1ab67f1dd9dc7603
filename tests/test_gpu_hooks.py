"""Device hook registry: the Zhang-Shu post-step kernel against its host
restatement on identical states (1D, 2D affine, 2D wavy), and its place in
the device time loop against a host-driven loop of single steps with the
host hook in between."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200.batch import Batch
from frforge_b200.limiters import zhang_shu_limit_

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


def test_batch_refuses_hook_methods():
    orc, state, _ = pair_2d(p=2, nx=4, ny=4)
    b = Batch(capacity=1)
    with pytest.raises(F.UnsupportedHookError):
        b.add(state, F.Euler2D(1.4), F.PositivityPreservingPersson())
    b.close()
