"""The preprocess_state hook slot on the GPU.

PositivityPreprocessPersson is a src/methods-style plugin whose
preprocess_state! limits the work state u_work with the Zhang-Shu scaling;
the residual (its sensor and dissipation included) is evaluated on u_work,
while the SSP-RK combination keeps the stage state, as in the reference's
residual! (Residual2D.jl:148) and ssp_rk3_step!.  The checks:

* the GPU residual with the hook equals the oracle's residual (identical
  inputs: the reference's tables) of the work state, which the device's own
  limiter produces (the post-step kernel runs the same element function; the
  host restatement, frforge_b200.limiters, agrees with it to 1e-13), in 2D
  and 1D;
* six fixed-dt SSP-RK3 steps with the hook equal a host-driven loop that
  evaluates, at every stage, the oracle residual of the limited stage state
  and combines it with the unlimited stage state;
* on an admissible state the hook changes nothing: bit-identical to the
  method without it;
* the batched engine refuses an instance with the hook.
"""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200 import _lib as L
from frforge_b200.batch import Batch
from frforge_b200.limiters import zhang_shu_limit_

from pairs import four_quadrant_state, pair_1d, pair_2d, rel_linf, smooth_state_2d

pytestmark = pytest.mark.gpu


def _spoil_2d(u):
    u = u.copy()
    u[1, 2, 5, 0] = -0.04     # negative density
    u[0, 1, 9, 3] = 1e-3      # negative pressure
    u[2, 2, 14, 3] = 0.02
    return u


EPS = dict(eps_rho=0.05, eps_p=0.05)  # floors well above round-off, so the limited state is well conditioned


def _device_limited(state, eq, u, caller_ops=None, eps=None):
    """The Zhang-Shu scaling of u by the device's own element function (the
    post-step kernel runs the same code as the preprocess kernel)."""
    s = F.GpuSolve(state, eq, F.PositivityPreservingPersson(**(eps or EPS)), caller_ops=caller_ops)
    s.upload(u, 0.0)
    s.apply_post_step()
    out, _ = s.download()
    s.close()
    return out


def test_residual_2d_is_that_of_the_limited_work_state():
    orc, state, _ = pair_2d(p=3, nx=6, ny=5, flux="hllc", method="persson", bcs=("transmissive",) * 4,
                            caller_ops=True, gpu_metrics=True)
    eq = F.Euler2D(1.4)
    u = _spoil_2d(four_quadrant_state(orc, jump_scale=0.25))
    uw = _device_limited(state, eq, u, orc.ops())
    assert not np.array_equal(uw, u)
    s = F.GpuSolve(state, eq, F.PositivityPreprocessPersson(**EPS), caller_ops=orc.ops())
    s.upload(u, 0.0)
    got = s.residual()
    orc.set_state(uw)
    orc.t = 0.0
    assert rel_linf(got, orc.residual()) <= 1e-12
    # and the host restatement of the limiter gives the same work state
    state.u[...] = u
    zhang_shu_limit_(state, eq, **EPS)
    assert rel_linf(state.u, uw) <= 1e-13
    s.close()


def test_residual_1d_is_that_of_the_limited_work_state():
    orc, state, _ = pair_1d(p=4, nel=12, method="persson", caller_ops=True)
    eq = F.Euler1D(1.4)
    orc.ic_sod()
    u = orc.u.copy()
    u[2, 3, 0] = -0.01
    u[1, 8, 2] = 1e-4
    uw = _device_limited(state, eq, u, orc.ops())
    assert not np.array_equal(uw, u)
    s = F.GpuSolve(state, eq, F.PositivityPreprocessPersson(**EPS), caller_ops=orc.ops())
    s.upload(u, 0.0)
    got = s.residual()
    orc.set_state(uw)
    orc.t = 0.0
    assert rel_linf(got, orc.residual()) <= 1e-12
    s.close()


def test_fixed_dt_steps_match_a_host_driven_loop():
    # floors of 0.3 act at every stage on this state (a density dip to 0.1 and
    # two low-energy points) while its face traces stay positive; a harsher
    # spoil limits the solution points but the Lagrange extrapolation to the
    # faces still overshoots to a negative density, and the scheme (the
    # reference's included) diverges at once
    orc, state, _ = pair_2d(p=2, nx=8, ny=8, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    eq = F.Euler2D(1.4)
    eps = dict(eps_rho=0.3, eps_p=0.3)
    u0 = four_quadrant_state(orc, jump_scale=0.25)
    u0[1, 2, 5, 0] = 0.1
    u0[0, 1, 9, 3] = 0.8
    u0[2, 2, 14, 3] = 1.0
    assert not np.array_equal(_device_limited(state, eq, u0, eps=eps), u0)
    dt, nsteps = 2e-4, 6

    def L_of(us, t):
        orc.set_state(_device_limited(state, eq, us, eps=eps))
        orc.t = t
        return orc.residual()

    u, t = u0.copy(), 0.0
    for _ in range(nsteps):
        u1 = u + dt * L_of(u, t)
        u2 = 0.75 * u + 0.25 * (u1 + dt * L_of(u1, t + dt))
        u = u / 3.0 + (2.0 / 3.0) * (u2 + dt * L_of(u2, t + dt / 2.0))
        t += dt
    s = F.GpuSolve(state, eq, F.PositivityPreprocessPersson(**eps))
    s.upload(u0, 0.0)
    r = s.advance(1.0, dt=dt, max_steps=nsteps)
    got, tg = s.download()
    assert r["n_steps"] == nsteps and tg == pytest.approx(t, rel=1e-14)
    assert rel_linf(got, u) <= 1e-10
    s.close()


def test_admissible_state_is_unchanged_by_the_hook():
    orc, state, plain = pair_2d(p=3, nx=10, ny=6, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    u = smooth_state_2d(orc)
    s = F.GpuSolve(state, F.Euler2D(1.4), F.PositivityPreprocessPersson())
    for solve in (plain, s):
        solve.upload(u, 0.0)
    assert np.array_equal(s.residual(), plain.residual())
    ra = plain.advance(1.0, cfl=0.1, max_steps=10)
    rb = s.advance(1.0, cfl=0.1, max_steps=10)
    assert ra == rb
    assert np.array_equal(s.download()[0], plain.download()[0])
    s.close()


def test_batch_refuses_the_hook():
    orc, state, _ = pair_2d(p=2, nx=8, ny=8, method="persson")
    b = Batch(capacity=1)
    i = b.add(state, F.Euler2D(1.4), F.PositivityPreprocessPersson())
    b.upload(i, smooth_state_2d(orc), 0.0)
    with pytest.raises(L.UnsupportedHookError):
        b.start(i, 1.0, cfl=0.1, max_steps=2)
    b.close()
